"""GPU parity of the batched density (locden) and batched preconditioner
against the CPU oracle.

Density: rho = sum_o hfac_o |psi_o(r)|^2 on the ISF grid (sumrho.f90:472-577,
OpenCL/Density.c:37-55).  Preconditioner: the CG recurrence of
ocl_preconditioner_generic (OpenCL/Preconditioner.c:130-195), x0 = b =
D^-1/2 r (the host's precondition_preconditioner with the initial guess off,
wfn_opt/precond.f90:711-714).  Bars: FP64 1e-13 (density), 1e-12 (CG output,
whose recurrence amplifies rounding), FP32 1e-5.
"""
import numpy as np
import pytest

from wvlh.batch import Batch
from wvlh.keys import Locreg

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def region(N, per, seed, dens=0.5):
    rng = np.random.default_rng(seed)
    mf = rng.random(N[::-1]) < dens
    return Locreg.from_masks(np.ones(N[::-1], bool), mf, per, (0.45, 0.4, 0.5))


def desc(oracle, lr):
    return oracle.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)


def layout(b, lrs, orb_lr, rows):
    psi = np.zeros(b.psi_size)
    for o, row in enumerate(rows):
        psi[b.psi_offset(o):b.psi_offset(o) + lrs[orb_lr[o]].ncoeff] = row
    return psi


@pytest.mark.parametrize("dtype_name,tol", [("float64", 1e-13), ("float32", 1e-5)])
def test_density_matches_oracle(oracle, torch_cuda, wctx, dtype_name, tol):
    torch = torch_cuda
    lrs = [region((10, 9, 11), (1, 1, 1), 1), region((7, 8, 6), (0, 0, 0), 2)]
    orb_lr = np.array([0, 0, 0, 1, 1], np.int32)
    off = [0, lrs[0].nisf]
    pot_off = np.array([off[l] for l in orb_lr], np.int64)
    b = Batch(wctx, lrs, orb_lr, pot_off)
    rng = np.random.default_rng(3)
    rows = [rng.uniform(-1, 1, lrs[l].ncoeff) for l in orb_lr]
    hfac = rng.uniform(0.5, 2.0, len(orb_lr))
    dt = getattr(torch, dtype_name)
    psi = torch.tensor(layout(b, lrs, orb_lr, rows), dtype=dt, device="cuda")
    rho = torch.full((lrs[0].nisf + lrs[1].nisf,), 1e-20, dtype=torch.float64, device="cuda")
    b.locden(psi, hfac, rho)
    torch.cuda.synchronize()
    got = rho.cpu().numpy()
    for l in range(2):
        ref = np.full(lrs[l].nisf, 1e-20)
        for o in np.nonzero(orb_lr == l)[0]:
            ref = oracle.locden(desc(oracle, lrs[l]), rows[o][:lrs[l].nvctr_c], rows[o][lrs[l].nvctr_c:],
                                hfac[o], ref)
        assert rel(got[off[l]:off[l] + lrs[l].nisf], ref) < tol


def test_density_many_orbitals_deterministic(torch_cuda, wctx):
    """64 orbitals sharing one grid are split in chunks; the fixed-order
    reduction makes repeated calls bit-identical."""
    torch = torch_cuda
    lr = region((12, 12, 12), (1, 1, 1), 4, 1.0)
    b = Batch(wctx, [lr], np.zeros(64, np.int32))
    psi = torch.rand(b.psi_size, dtype=torch.float64, device="cuda") - 0.5
    r1 = torch.zeros(lr.nisf, dtype=torch.float64, device="cuda")
    r2 = torch.zeros_like(r1)
    hf = np.full(64, 2.0)
    b.locden(psi, hf, r1)
    b.locden(psi, hf, r2)
    torch.cuda.synchronize()
    assert torch.equal(r1, r2)
    assert (r1 > 0).all()


@pytest.mark.parametrize("dtype_name,tol", [("float64", 1e-12), ("float32", 1e-5)])
def test_preconditioner_matches_oracle(oracle, torch_cuda, wctx, dtype_name, tol):
    torch = torch_cuda
    lrs = [region((10, 9, 11), (1, 1, 1), 5), region((7, 8, 6), (0, 0, 0), 6)]
    orb_lr = np.array([0, 0, 1], np.int32)
    b = Batch(wctx, lrs, orb_lr)
    rng = np.random.default_rng(7)
    cprec = np.array([0.7, 1.3, 0.9])
    xs, bs = [], []
    for o, l in enumerate(orb_lr):
        lr = lrs[l]
        r = rng.uniform(-1, 1, lr.ncoeff)
        s = oracle.precond_scal([0.5 * h for h in lr.hgrid], cprec[o])
        sc = np.concatenate([np.full(lr.nvctr_c, s[0]), np.tile(s[1:], lr.nvctr_f)])
        xs.append(sc * r)
        bs.append(sc * r)
    dt = getattr(torch, dtype_name)
    x = torch.tensor(layout(b, lrs, orb_lr, xs), dtype=dt, device="cuda")
    rhs = torch.tensor(layout(b, lrs, orb_lr, bs), dtype=dt, device="cuda")
    x, hist = b.precond(x, rhs, cprec, 5)
    torch.cuda.synchronize()
    xg = x.double().cpu().numpy()
    hist = hist.cpu().numpy()
    for o, l in enumerate(orb_lr):
        lr = lrs[l]
        ref, rn = oracle.precond(desc(oracle, lr), [0.5 * h for h in lr.hgrid], cprec[o], 5, xs[o], bs[o])
        got = xg[b.psi_offset(o):b.psi_offset(o) + lr.ncoeff]
        assert rel(got, ref) < tol
        assert np.allclose(hist[:, o], rn, rtol=10 * tol, atol=0)
        assert hist[-1, o] < hist[0, o]      # the CG reduces the residual


@pytest.mark.parametrize("dtype_name,tol", [("float64", 1e-13), ("float32", 1e-5)])
def test_density_long_z_pencils(oracle, torch_cuda, wctx, dtype_name, tol):
    """Free box with 52 coarse cells along z: ISF z-length 133 > 128 takes the
    density kernel's 48-accumulator variant."""
    torch = torch_cuda
    lr = region((9, 8, 52), (0, 0, 0), 8, 0.4)
    b = Batch(wctx, [lr], np.zeros(3, np.int32))
    rng = np.random.default_rng(9)
    rows = [rng.uniform(-1, 1, lr.ncoeff) for _ in range(3)]
    hfac = rng.uniform(0.5, 2.0, 3)
    dt = getattr(torch, dtype_name)
    psi = torch.tensor(layout(b, [lr], [0, 0, 0], rows), dtype=dt, device="cuda")
    rho = torch.zeros(lr.nisf, dtype=torch.float64, device="cuda")
    b.locden(psi, hfac, rho)
    torch.cuda.synchronize()
    ref = np.zeros(lr.nisf)
    for o in range(3):
        ref = oracle.locden(desc(oracle, lr), rows[o][:lr.nvctr_c], rows[o][lr.nvctr_c:], hfac[o], ref)
    assert rel(rho.cpu().numpy(), ref) < tol


@pytest.mark.parametrize("dtype_name", ["float64", "float32"])
def test_precond_autotune_keeps_results(torch_cuda, wctx, dtype_name):
    """wvlh_batch_autotune_precond times each compiled block size of the plane
    kernels on the batch's own preconditioner and keeps the fastest; the
    preconditioned vectors depend on the pick only through the summation order
    of <d|Ad>, which K3 accumulates per thread while it scatters A d."""
    torch = torch_cuda
    lrs = [region((10, 9, 11), (1, 1, 1), 5), region((7, 8, 6), (0, 0, 0), 6)]
    orb_lr = np.array([0, 1, 0], np.int32)
    b = Batch(wctx, lrs, orb_lr)
    rng = np.random.default_rng(12)
    cprec = np.array([0.8, 1.1, 0.6])
    dt = getattr(torch, dtype_name)
    rhs = torch.tensor(rng.uniform(-1, 1, b.psi_size), dtype=dt, device="cuda")
    x0, h0 = b.precond(rhs.clone(), rhs, cprec, 3)
    x0, h0 = x0.clone(), h0.clone()
    pick, times = b.autotune_precond(rhs.clone(), rhs, cprec, 3, reps=1)
    assert pick in times and len(times) >= 4 and all(t > 0 for t in times.values())
    bs = b.block_sizes()["precond"]
    assert bs["plane"][0 if dtype_name == "float32" else 1] == pick and bs["z"][0] in (256, 320, 384)
    x1, h1 = b.precond(rhs.clone(), rhs, cprec, 3)
    torch.cuda.synchronize()
    tol = 1e-13 if dtype_name == "float64" else 1e-5
    assert ((x1.double() - x0.double()).norm() / x0.double().norm()).item() <= tol
    assert ((h1 - h0).abs() / h0.abs()).max().item() <= 10 * tol
    x2, h2 = b.precond(rhs.clone(), rhs, cprec, 3)
    torch.cuda.synchronize()
    assert torch.equal(x2, x1) and torch.equal(h2, h1)   # deterministic for a given block size
    b.close()


@pytest.mark.parametrize("N,per", [((64, 64, 8), (1, 1, 1)), ((48, 46, 6), (0, 0, 0))])
def test_precond_large_planes_match_oracle(oracle, torch_cuda, wctx, N, per):
    """FP64 boxes whose two planes exceed a block's shared memory keep the
    second plane in a global slice per CTA: the CG direction update and the
    <d|Ad> staging then go through that slice instead of shared memory."""
    torch = torch_cuda
    lr = region(N, per, 13, 0.5)
    b = Batch(wctx, [lr, lr], np.zeros(2, np.int32))
    rng = np.random.default_rng(14)
    cprec = np.array([0.8, 1.2])
    rows = [rng.uniform(-1, 1, lr.ncoeff) for _ in range(2)]
    x = torch.tensor(layout(b, [lr], [0, 0], rows), dtype=torch.float64, device="cuda")
    rhs = x.clone()
    x, hist = b.precond(x, rhs, cprec, 3)
    torch.cuda.synchronize()
    xg, hist = x.cpu().numpy(), hist.cpu().numpy()
    for o in range(2):
        ref, rn = oracle.precond(desc(oracle, lr), [0.5 * h for h in lr.hgrid], cprec[o], 3, rows[o], rows[o])
        assert rel(xg[b.psi_offset(o):b.psi_offset(o) + lr.ncoeff], ref) < 1e-13
        assert np.allclose(hist[:, o], rn, rtol=1e-12, atol=0)
