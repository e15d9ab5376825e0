"""GPU parity of the batched local Hamiltonian against the CPU oracle.

Bars: FP64 paths within 1e-13 relative L2 of the oracle on Hpsi and 1e-12
relative on the energies (the reference's own GPU-vs-CPU tolerance is 1e-9 to
2.6e-10, bigdft/tests/libs/OpenCL/tols.yaml); FP32 forms within 1e-6 Ha on
E_kin / E_pot per normalised orbital and 1e-5 relative L2 on Hpsi.
"""
from pathlib import Path

import numpy as np
import pytest

from wvlh import workloads as W
from wvlh.batch import Batch
from wvlh.keys import Locreg

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def case(N, per, density=0.5, seed=0, hgrid=(0.45, 0.4, 0.5), empty_fine=False):
    rng = np.random.default_rng(seed)
    mc = np.ones(N[::-1], bool)
    mf = np.zeros(N[::-1], bool) if empty_fine else (rng.random(N[::-1]) < density)
    lr = Locreg.from_masks(mc, mf, per, hgrid)
    psi = rng.uniform(-1, 1, lr.ncoeff)
    pot = rng.uniform(-1, 0, lr.nisf)
    return lr, psi, pot


def oracle_locham(oracle, lr, psi, pot):
    d = oracle.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
    hc, hf, ek, ep = oracle.locham(d, lr.hgrid, psi[:lr.nvctr_c], psi[lr.nvctr_c:], pot)
    return np.concatenate([hc, hf]), ek, ep


def run_batch(wctx, torch, lrs, psis, pots, dtype, plain=False):
    """One orbital per region, each with its own potential."""
    pot_off = np.cumsum([0] + [lr.nisf for lr in lrs[:-1]])
    b = Batch(wctx, lrs, np.arange(len(lrs)), pot_off)
    psi = np.zeros(b.psi_size)
    for o, p in enumerate(psis):
        psi[b.psi_offset(o):b.psi_offset(o) + len(p)] = p
    tp = torch.tensor(psi, dtype=dtype, device="cuda")
    tv = torch.tensor(np.concatenate(pots), dtype=dtype, device="cuda")
    if plain:
        h, ek, ep = b.locham_plain(tp, tv)
    else:
        h, ek, ep = b.locham(tp, tv)
    torch.cuda.synchronize()
    h = h.double().cpu().numpy()
    out = [h[b.psi_offset(o):b.psi_offset(o) + lrs[o].ncoeff] for o in range(len(lrs))]
    return out, ek.cpu().numpy(), ep.cpu().numpy()


CASES = [
    ((8, 9, 10), (1, 1, 1), 0.5, False),
    ((16, 16, 16), (1, 1, 1), 1.0, False),
    ((11, 8, 13), (1, 1, 1), 0.3, False),
    ((6, 7, 5), (0, 0, 0), 0.5, False),
    ((12, 10, 9), (0, 0, 0), 0.7, False),
    ((8, 6, 8), (1, 0, 1), 0.5, False),
    ((9, 8, 8), (1, 1, 1), 0.0, True),     # no fine region (nseg_f = 0)
    ((5, 5, 5), (0, 0, 0), 0.0, True),
]


@pytest.mark.parametrize("N,per,dens,empty", CASES)
@pytest.mark.parametrize("plain", [False, True])
def test_fp64_matches_oracle(oracle, torch_cuda, wctx, N, per, dens, empty, plain):
    lr, psi, pot = case(N, per, dens, seed=hash((N, per)) % 1000, empty_fine=empty)
    ref, ek, ep = oracle_locham(oracle, lr, psi, pot)
    out, gek, gep = run_batch(wctx, torch_cuda, [lr], [psi], [pot], torch_cuda.float64, plain=plain)
    assert rel(out[0], ref) < 1e-13
    assert abs(gek[0] - ek) <= 1e-12 * abs(ek) and abs(gep[0] - ep) <= 1e-12 * abs(ep)


def test_heterogeneous_batch_fp64_and_fp32(oracle, torch_cuda, wctx):
    cs = [case(N, per, d, seed=i) for i, (N, per, d, _) in enumerate(CASES[:6])]
    lrs, psis, pots = zip(*cs)
    psis = [p / np.linalg.norm(p) for p in psis]
    refs = [oracle_locham(oracle, lr, p, v) for lr, p, v in zip(lrs, psis, pots)]
    out, ek, ep = run_batch(wctx, torch_cuda, list(lrs), psis, list(pots), torch_cuda.float64)
    for o, (r, e1, e2) in enumerate(refs):
        assert rel(out[o], r) < 1e-13
        assert abs(ek[o] - e1) <= 1e-12 * abs(e1) and abs(ep[o] - e2) <= 1e-12 * abs(e2)
    out, ek, ep = run_batch(wctx, torch_cuda, list(lrs), psis, list(pots), torch_cuda.float32)
    for o, (r, e1, e2) in enumerate(refs):
        assert rel(out[o], r) < 1e-5
        assert abs(ek[o] - e1) < 1e-6 and abs(ep[o] - e2) < 1e-6


def test_golden_regression_vectors(torch_cuda, wctx):
    g = np.load(GOLD / "locham_small.npz")
    for name, N, per in (("per", (8, 9, 10), (1, 1, 1)), ("free", (6, 7, 5), (0, 0, 0)),
                         ("surf", (8, 6, 8), (1, 0, 1))):
        lr = Locreg.from_masks(np.ones(N[::-1], bool), g[name + "_mf"].astype(bool), per, (0.45, 0.4, 0.5))
        out, ek, ep = run_batch(wctx, torch_cuda, [lr], [g[name + "_psi"]], [g[name + "_pot"]], torch_cuda.float64)
        assert rel(out[0], g[name + "_hpsi"]) < 1e-13
        assert np.allclose([ek[0], ep[0]], g[name + "_e"], rtol=1e-12, atol=0)


def test_accumulate_and_host_entry(oracle, torch_cuda, wctx):
    lr, psi, pot = case((8, 8, 9), (1, 1, 1), 0.6, seed=11)
    ref, ek, ep = oracle_locham(oracle, lr, psi, pot)
    b = Batch(wctx, [lr], [0])
    tp = torch_cuda.tensor(psi, device="cuda")
    tv = torch_cuda.tensor(pot, device="cuda")
    base = torch_cuda.full_like(tp, 0.25)
    h, _, _ = b.locham(tp, tv, hpsi=base.clone(), accumulate=True)
    assert rel(h.cpu().numpy() - 0.25, ref) < 1e-13
    hh = np.zeros_like(psi)
    e1, e2 = np.zeros(1), np.zeros(1)
    b.locham_host(psi, pot, hh, e1, e2, 64)
    assert rel(hh, ref) < 1e-13 and abs(e1[0] - ek) <= 1e-12 * abs(ek)


@pytest.mark.parametrize("dtype_name", ["float32", "float64"])
def test_host_entry_in_chunks_matches_device_entry(torch_cuda, wctx, dtype_name):
    """Batches of 8 orbitals or more go through the host-buffer entry point in
    chunks on two streams: the same kernels per orbital, so the same bits."""
    torch = torch_cuda
    lrs = [case((10, 9, 12), (1, 1, 1), 0.6, seed=21)[0], case((9, 8, 7), (0, 0, 0), 0.5, seed=22)[0]]
    orb_lr = np.array([0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 1, 0, 0], np.int32)
    off = np.cumsum([0] + [lr.nisf for lr in lrs])
    b = Batch(wctx, lrs, orb_lr, off[orb_lr])
    rng = np.random.default_rng(4)
    dt = np.float32 if dtype_name == "float32" else np.float64
    psi = rng.uniform(-1, 1, b.psi_size).astype(dt)
    pot = rng.uniform(-1, 0, int(off[-1])).astype(dt)
    hd, ekd, epd = b.locham(torch.tensor(psi, device="cuda"), torch.tensor(pot, device="cuda"))
    torch.cuda.synchronize()
    hh = np.zeros_like(psi)
    e1, e2 = np.zeros(len(orb_lr)), np.zeros(len(orb_lr))
    for _ in range(2):   # the second call reuses the chunks
        b.locham_host(psi, pot, hh, e1, e2, 32 if dt == np.float32 else 64)
        assert np.array_equal(hh, hd.cpu().numpy())
        assert np.array_equal(e1, ekd.cpu().numpy()) and np.array_equal(e2, epd.cpu().numpy())


@pytest.mark.parametrize("dtype_name", ["float32", "float64"])
def test_graph_replay_matches_direct_call(torch_cuda, wctx, dtype_name):
    """A captured locham replays the same kernels: the same bits, and it reads
    the buffers' current contents at every launch."""
    torch = torch_cuda
    lrs = [case((10, 9, 12), (1, 1, 1), 0.6, seed=31)[0], case((9, 8, 7), (0, 0, 0), 0.5, seed=32)[0]]
    orb_lr = np.array([0, 1, 1, 0, 0], np.int32)
    off = np.cumsum([0] + [lr.nisf for lr in lrs])
    b = Batch(wctx, lrs, orb_lr, off[orb_lr])
    dt = getattr(torch, dtype_name)
    g = torch.Generator(device="cuda").manual_seed(5)
    psi = torch.rand(b.psi_size, generator=g, device="cuda", dtype=torch.float64).to(dt) - 0.5
    pot = -torch.rand(int(off[-1]), generator=g, device="cuda", dtype=torch.float64).to(dt)
    h1, e1, p1 = b.locham(psi, pot)
    h2, e2, p2 = torch.zeros_like(h1), torch.zeros_like(e1), torch.zeros_like(p1)
    graph = b.locham_graph(psi, pot, h2, e2, p2)
    for _ in range(2):
        graph.launch()
        torch.cuda.synchronize()
        assert torch.equal(h1, h2) and torch.equal(e1, e2) and torch.equal(p1, p2)
    psi.mul_(2)
    h3, e3, p3 = b.locham(psi, pot)
    graph.launch()
    torch.cuda.synchronize()
    assert torch.equal(h3, h2) and torch.equal(e3, e2)
    graph.close()


def test_invalid_keys_rejected(torch_cuda, wctx):
    from wvlh._lib import WvlhError
    lr, _, _ = case((8, 8, 8), (1, 1, 1), 0.5, seed=3)
    bad = Locreg(lr.n, lr.periodic, lr.hgrid, lr.keyg_c.copy(), lr.keyv_c.copy(), lr.keyg_f, lr.keyv_f)
    bad.keyg_c[3, 1] = bad.keyg_c[3, 0] + 20  # crosses an x-line
    with pytest.raises(WvlhError, match="keys"):
        Batch(wctx, [bad], [0])
    bad2 = Locreg(lr.n, lr.periodic, lr.hgrid, lr.keyg_c, lr.keyv_c.copy(), lr.keyg_f, lr.keyv_f)
    bad2.keyv_c[5] += 1  # compressed offsets inconsistent with segment lengths
    with pytest.raises(WvlhError, match="keys"):
        Batch(wctx, [bad2], [0])


def test_full_size_properties_fp32_vs_fp64(torch_cuda, wctx):
    """48^3 periodic box (the batched configuration's grid), 16 normalised
    orbitals: FP32 energies within 1e-6 Ha of FP64, FP64 Hermiticity, linearity."""
    lr, psi, pot = W.batched_periodic(n=48, norb=16, seed=5)
    b = Batch(wctx, [lr], np.zeros(16, np.int32))
    t64 = torch_cuda.tensor(psi.ravel(), device="cuda")
    v64 = torch_cuda.tensor(pot, device="cuda")
    h64, ek64, ep64 = b.locham(t64, v64)
    h32, ek32, ep32 = b.locham(t64.float(), v64.float())
    torch_cuda.cuda.synchronize()
    assert (ek32 - ek64).abs().max().item() < 1e-6
    assert (ep32 - ep64).abs().max().item() < 1e-6
    H = h64.view(16, -1)
    P = t64.view(16, -1)
    M = P @ H.T                       # <psi_i|H|psi_j>
    assert ((M - M.T).abs().max() / M.abs().max()).item() < 1e-13
    # diagonal equals ekin + epot
    assert ((M.diagonal() - (ek64 + ep64)).abs().max() / M.diagonal().abs().max()).item() < 1e-13
    # linearity: H(a x + y) = a Hx + Hy
    hx, _, _ = b.locham((2.5 * P[0:1] + P[1:2]).repeat(16, 1).ravel().contiguous(), v64)
    assert ((hx.view(16, -1)[0] - (2.5 * H[0] + H[1])).norm() / H[0].norm()).item() < 1e-13


# FP64 planes too large for two shared-memory buffers (2 x rows x pitch x 8 B
# above the 227 KB per block): the second buffer is a global slice per CTA.
LARGE = [((48, 46, 6), (0, 0, 0), 0.5), ((64, 64, 8), (1, 1, 1), 1.0), ((60, 62, 9), (0, 0, 0), 0.4)]


@pytest.mark.parametrize("N,per,dens", LARGE)
def test_fp64_large_planes_match_oracle(oracle, torch_cuda, wctx, N, per, dens):
    lr, psi, pot = case(N, per, dens, seed=5)
    psi /= np.linalg.norm(psi)
    ref, ek, ep = oracle_locham(oracle, lr, psi, pot)
    out, gek, gep = run_batch(wctx, torch_cuda, [lr, lr], [psi, psi], [pot, pot], torch_cuda.float64)
    for o in range(2):
        assert rel(out[o], ref) < 1e-13
        assert abs(gek[o] - ek) <= 1e-12 * abs(ek) and abs(gep[o] - ep) <= 1e-12 * abs(ep)
    # the FP32 form of the same boxes keeps two shared planes
    out, gek, gep = run_batch(wctx, torch_cuda, [lr], [psi], [pot], torch_cuda.float32)
    assert rel(out[0], ref) < 1e-5 and abs(gek[0] - ek) < 1e-6 and abs(gep[0] - ep) < 1e-6


@pytest.mark.parametrize("dtype_name,tol", [("float64", 1e-13), ("float32", 1e-6)])
def test_autotune_times_every_block_size_and_keeps_results(oracle, torch_cuda, wctx, dtype_name, tol):
    """wvlh_batch_autotune times each compiled block size of the plane kernels
    (then, FP32, of the z kernel) on the batch's own locham and keeps the
    fastest; Hpsi does not depend on the pick, the energies only through their
    summation order (FP32: the z kernel's per-thread partial sums of E_pot
    change with its block size, an FP32-rounding difference)."""
    torch = torch_cuda
    lrs = [case((12, 10, 9), (0, 0, 0), 0.6, seed=1)[0], case((10, 11, 12), (1, 1, 1), 0.5, seed=2)[0]]
    rng = np.random.default_rng(4)
    b = Batch(wctx, lrs, [0, 1, 1], np.cumsum([0] + [lrs[0].nisf, lrs[1].nisf])[:3])
    dt = getattr(torch, dtype_name)
    psi = torch.tensor(rng.uniform(-1, 1, b.psi_size), dtype=dt, device="cuda")
    pot = torch.tensor(rng.uniform(-1, 0, b.pot_size), dtype=dt, device="cuda")
    h0, e0, p0 = b.locham(psi, pot)
    h0, e0, p0 = h0.clone(), e0.clone(), p0.clone()
    pick, times = b.autotune(psi, pot, reps=1)
    assert pick in times and len(times) >= 4 and all(t > 0 for t in times.values())
    bs = b.block_sizes()["locham"]
    assert bs["plane"][0 if dtype_name == "float32" else 1] == pick
    assert bs["z"][0] in (256, 320, 384) and bs["z"][1] == 256
    h1, e1, p1 = b.locham(psi, pot)
    torch.cuda.synchronize()
    assert ((h1 - h0).norm() / h0.norm()).item() <= tol
    etol = 1e-12 if dtype_name == "float64" else 1e-7
    assert ((e1 - e0).abs() / e0.abs()).max().item() <= etol and ((p1 - p0).abs() / p0.abs()).max().item() <= etol
    b.close()
