"""GPU-vs-oracle parity at the full sizes of the five benchmark workloads.

* single orbital: periodic 32^3 coarse (64^3 fine), one orbital of uniform(-1,1)
  coefficients, hgrid 0.45, 4-Gaussian potential; FP64 fused and plain paths
  within 1e-13 relative L2 on Hpsi and 1e-12 relative on E_kin / E_pot;
* batched: 256 normalised orbitals on one periodic 48^3 grid; the whole batch
  runs in one launch and 4 of its orbitals are compared with the oracle
  (FP64 1e-13 / 1e-12; FP32 1e-5 relative L2 on Hpsi and 1e-6 Ha on the
  energies), plus the density of 8 orbitals and the 256 x 256 overlap;
* free regions: 8 regions of the free-BC generator (coarse 20..40 per
  dimension, fine ellipsoid of radius 0.4 x the box), one launch;
* preconditioner: 40^3 periodic, 5 CG iterations of (T - eps + c) x = r with
  x0 = b = r, c = 0.5, eps uniform(-1, -0.1); x and the squared residual norm
  of every iteration against the oracle (FP64 1e-12 / FP32 1e-5);
* serving: the largest periodic and the largest free client box of the
  serving workload, through per-orbital buffers (orbital batches).

The oracle is the FP64 C restatement of the reference's CPU chain
(orbitals/convolut_simple_per.f90, wavelib/un-compress.f90,
orbitals/potential.f90, sumrho.f90, wfn_opt/precond.f90).
"""
import numpy as np
import pytest

from wvlh import workloads as W
from wvlh.batch import Batch, OrbitalBatch, Region

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def desc(oracle, lr):
    return oracle.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)


def oracle_locham(oracle, lr, psi, pot):
    hc, hf, ek, ep = oracle.locham(desc(oracle, lr), lr.hgrid, psi[:lr.nvctr_c], psi[lr.nvctr_c:], pot)
    return np.concatenate([hc, hf]), ek, ep


@pytest.mark.parametrize("plain", [False, True])
def test_single_orbital_32cubed_fp64(oracle, torch_cuda, wctx, plain):
    torch = torch_cuda
    lr, psi, pot = W.single_orbital(32, seed=0)
    ref, ek, ep = oracle_locham(oracle, lr, psi, pot)
    b = Batch(wctx, [lr], [0])
    tp = torch.tensor(psi, device="cuda")
    tv = torch.tensor(pot, device="cuda")
    h, gek, gep = b.locham_plain(tp, tv) if plain else b.locham(tp, tv)
    torch.cuda.synchronize()
    assert rel(h.cpu().numpy(), ref) < 1e-13
    assert abs(gek[0].item() - ek) <= 1e-12 * abs(ek)
    assert abs(gep[0].item() - ep) <= 1e-12 * abs(ep)
    b.close()


@pytest.fixture(scope="module")
def batched48(torch_cuda, wctx):
    """The batched workload on the device, as the benchmark builds it."""
    torch = torch_cuda
    lr, psi, pot = W.batched_periodic_device(torch, "cuda", n=48, norb=256, seed=1000)
    b = Batch(wctx, [lr], np.zeros(256, np.int32))
    yield lr, psi, pot, b
    b.close()


SAMPLE = [0, 77, 190, 255]


@pytest.mark.parametrize("prec", [64, 32])
def test_batched_48cubed_256_orbitals(oracle, torch_cuda, batched48, prec):
    torch = torch_cuda
    lr, psi, pot, b = batched48
    dt = torch.float64 if prec == 64 else torch.float32
    h, ek, ep = b.locham(psi.to(dt), pot.to(dt))
    torch.cuda.synchronize()
    P = psi.view(256, -1)
    H = h.view(256, -1)
    vh = pot.cpu().numpy()
    for o in SAMPLE:
        x = P[o].cpu().numpy()
        ref, e1, e2 = oracle_locham(oracle, lr, x, vh)
        got = H[o].double().cpu().numpy()
        if prec == 64:
            assert rel(got, ref) < 1e-13
            assert abs(ek[o].item() - e1) <= 1e-12 * abs(e1) and abs(ep[o].item() - e2) <= 1e-12 * abs(e2)
        else:
            assert rel(got, ref) < 1e-5
            assert abs(ek[o].item() - e1) < 1e-6 and abs(ep[o].item() - e2) < 1e-6


@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 1e-5)])
def test_batched_48cubed_density_and_overlap(oracle, torch_cuda, wctx, batched48, prec, tol):
    torch = torch_cuda
    lr, psi, pot, _ = batched48
    P = psi.view(256, -1)
    # density of 8 of the orbitals (occupation 2 over the fine-grid cell volume)
    b8 = Batch(wctx, [lr], np.zeros(8, np.int32))
    dt = torch.float64 if prec == 64 else torch.float32
    sub = P[SAMPLE + [1, 2, 3, 4]].contiguous()
    vol = np.prod([0.5 * h for h in lr.hgrid])
    hfac = np.full(8, 2.0 / vol)
    rho = torch.zeros(lr.nisf, dtype=torch.float64, device="cuda")
    b8.locden(sub.reshape(-1).to(dt), hfac, rho)
    torch.cuda.synchronize()
    ref = np.zeros(lr.nisf)
    for o in range(8):
        x = sub[o].cpu().numpy()
        ref = oracle.locden(desc(oracle, lr), x[:lr.nvctr_c], x[lr.nvctr_c:], hfac[o], ref)
    assert rel(rho.cpu().numpy(), ref) < tol
    b8.close()
    if prec == 64:
        from wvlh.ortho import overlap
        S = overlap(wctx, P).cpu().numpy()
        Ph = P.cpu().numpy()
        Sref = Ph @ Ph.T
        assert np.abs(S - Sref).max() < 1e-13 * np.abs(Sref).max()


def test_free_regions_fp64_fp32(oracle, torch_cuda, wctx):
    torch = torch_cuda
    lrs, psis, pots = W.free_regions(nlr=8, seed=2)
    off = np.cumsum([0] + [lr.nisf for lr in lrs[:-1]])
    b = Batch(wctx, lrs, np.arange(8, dtype=np.int32), off)
    flat = np.zeros(b.psi_size)
    for o, p in enumerate(psis):
        flat[b.psi_offset(o):b.psi_offset(o) + len(p)] = p
    refs = [oracle_locham(oracle, lr, p, v) for lr, p, v in zip(lrs, psis, pots)]
    for dt in (torch.float64, torch.float32):
        h, ek, ep = b.locham(torch.tensor(flat, dtype=dt, device="cuda"),
                             torch.tensor(np.concatenate(pots), dtype=dt, device="cuda"))
        torch.cuda.synchronize()
        h = h.double().cpu().numpy()
        for o, (r, e1, e2) in enumerate(refs):
            got = h[b.psi_offset(o):b.psi_offset(o) + lrs[o].ncoeff]
            if dt == torch.float64:
                assert rel(got, r) < 1e-13
                assert abs(ek[o].item() - e1) <= 1e-12 * abs(e1) and abs(ep[o].item() - e2) <= 1e-12 * abs(e2)
            else:
                assert rel(got, r) < 1e-5
                assert abs(ek[o].item() - e1) < 1e-6 and abs(ep[o].item() - e2) < 1e-6
    b.close()


@pytest.mark.parametrize("prec,tol", [(64, 1e-12), (32, 1e-5)])
def test_precond_40cubed(oracle, torch_cuda, wctx, prec, tol):
    torch = torch_cuda
    lr = W.full_periodic(40, 0.45)
    norb = 4
    rng = np.random.default_rng(3)
    cprec = 0.5 - rng.uniform(-1.0, -0.1, norb)
    r = rng.uniform(-1, 1, (norb, lr.ncoeff))
    b = Batch(wctx, [lr], np.zeros(norb, np.int32))
    dt = torch.float64 if prec == 64 else torch.float32
    rt = torch.tensor(r.ravel(), dtype=dt, device="cuda")
    x, hist = b.precond(rt.clone(), rt, cprec, 5)
    torch.cuda.synchronize()
    xg = x.double().cpu().numpy().reshape(norb, -1)
    hist = hist.cpu().numpy()
    hf = [0.5 * h for h in lr.hgrid]
    for o in range(norb):
        ref, rn = oracle.precond(desc(oracle, lr), hf, cprec[o], 5, r[o], r[o])
        assert rel(xg[o], ref) < tol
        assert np.allclose(hist[:, o], rn, rtol=10 * tol, atol=0)
    b.close()


def test_serving_client_boxes(oracle, torch_cuda, wctx):
    torch = torch_cuda
    specs = W.serving_clients()
    per = max((s for s in specs if all(s[0].periodic)), key=lambda s: s[0].coarse_cells)[0]
    free = max((s for s in specs if not any(s[0].periodic)), key=lambda s: s[0].coarse_cells)[0]
    rng = np.random.default_rng(8)
    items, refs = [], []
    for lr in (per, free):
        psi = W.random_psi(lr, 1, rng, normalize=True)[0]
        pot = W.gaussian_potential(lr, rng)
        reg = Region(wctx, lr)
        items.append((reg, torch.tensor(psi, device="cuda"), torch.zeros(lr.ncoeff, dtype=torch.float64,
                                                                          device="cuda"),
                      torch.tensor(pot, device="cuda"), None))
        refs.append(oracle_locham(oracle, lr, psi, pot))
    ob = OrbitalBatch(wctx, items)
    ek = torch.empty(2, dtype=torch.float64, device="cuda")
    ep = torch.empty_like(ek)
    ob.locham(ek, ep)
    torch.cuda.synchronize()
    for o, (r, e1, e2) in enumerate(refs):
        assert rel(items[o][2].cpu().numpy(), r) < 1e-13
        assert abs(ek[o].item() - e1) <= 1e-12 * abs(e1) and abs(ep[o].item() - e2) <= 1e-12 * abs(e2)
    ob.close()
    for it in items:
        it[0].close()
