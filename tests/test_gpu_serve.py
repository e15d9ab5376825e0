"""Serving on the GPU: resident regions, orbital batches over many clients'
own buffers, and the continuous-batching server of wvlh.serve.

The bar of the mix test: each client's result (hpsi, energies, density) is
the same alone and in the mix.  A batch of periodic clients only runs the
periodic-specialised kernels, a mixed one the generic kernels, so the two may
differ by rounding: FP64 within 1e-13 relative L2 (energies 1e-12 relative),
FP32 within 1e-6 relative L2 (energies 1e-6 Ha).  Orbital batches and packed
batches over the same orbitals are bit-identical (same kernels, same order).
"""
import numpy as np
import pytest

from wvlh._lib import WvlhError
from wvlh.batch import Batch, OrbitalBatch, Region
from wvlh.serve import Server, latency_stats, request_scratch
from wvlh.workloads import free_sphere, full_periodic, gaussian_potential, poisson_arrivals

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def small_clients():
    return [(full_periodic((16, 12, 10)), 5), (free_sphere((11, 13, 9)), 3), (full_periodic((8, 9, 12)), 4),
            (free_sphere((14, 10, 12)), 6), (free_sphere((9, 9, 9)), 2)]


def client_data(lr, norb, seed):
    rng = np.random.default_rng(seed)
    psi = rng.uniform(-1, 1, (norb, lr.ncoeff))
    psi /= np.linalg.norm(psi, axis=1, keepdims=True)
    return psi, gaussian_potential(lr, rng)


@pytest.mark.parametrize("dtype_name", ["float64", "float32"])
def test_orbital_batch_bit_identical_to_packed(torch_cuda, wctx, dtype_name):
    torch = torch_cuda
    dt = getattr(torch, dtype_name)
    lrs = [lr for lr, _ in small_clients()[:3]]
    orb_lr = np.array([0, 1, 0, 2, 1, 2, 2], np.int32)
    rng = np.random.default_rng(7)
    rows = [rng.uniform(-1, 1, lrs[l].ncoeff) for l in orb_lr]
    pots = [gaussian_potential(lr, rng) for lr in lrs]
    hfac = rng.uniform(0.5, 2.0, len(orb_lr))
    # packed: one psi array, potentials at offsets, densities at the same offsets
    off = np.cumsum([0] + [lr.nisf for lr in lrs])
    b = Batch(wctx, lrs, orb_lr, off[orb_lr])
    psi = np.zeros(b.psi_size)
    for o, r in enumerate(rows):
        psi[b.psi_offset(o):b.psi_offset(o) + len(r)] = r
    psi_t = torch.tensor(psi, dtype=dt, device="cuda")
    pot_t = torch.tensor(np.concatenate(pots), dtype=dt, device="cuda")
    hp, ek, ep = b.locham(psi_t, pot_t)
    rho = torch.zeros(int(off[-1]), dtype=torch.float64, device="cuda")
    b.locden(psi_t, hfac, rho)
    # orbital batch: every orbital and region with its own allocations
    regs = [Region(wctx, lr) for lr in lrs]
    psi_o = [torch.tensor(r, dtype=dt, device="cuda") for r in rows]
    hpsi_o = [torch.zeros_like(p) for p in psi_o]
    pot_o = [torch.tensor(p, dtype=dt, device="cuda") for p in pots]
    rho_o = [torch.zeros(lr.nisf, dtype=torch.float64, device="cuda") for lr in lrs]
    ob = OrbitalBatch(wctx, [(regs[l], psi_o[o], hpsi_o[o], pot_o[l], None) for o, l in enumerate(orb_lr)])
    ek2 = torch.empty(len(orb_lr), dtype=torch.float64, device="cuda")
    ep2 = torch.empty_like(ek2)
    ob.locham(ek2, ep2)
    ob.close()
    ob = OrbitalBatch(wctx, [(regs[l], psi_o[o], None, None, rho_o[l]) for o, l in enumerate(orb_lr)])
    ob.locden(torch.tensor(hfac, device="cuda"))
    torch.cuda.synchronize()
    for o in range(len(orb_lr)):
        n = len(rows[o])
        assert torch.equal(hpsi_o[o], hp[b.psi_offset(o):b.psi_offset(o) + n])
    assert torch.equal(ek, ek2) and torch.equal(ep, ep2)
    for l in range(len(lrs)):
        assert torch.equal(rho_o[l], rho[int(off[l]):int(off[l + 1])])
    for l, lr in enumerate(lrs):
        assert regs[l].scratch_bytes(64) == request_scratch(lr, 1, 8)
        assert regs[l].grid_size == lr.nisf and regs[l].psi_size == lr.ncoeff


def test_stale_orbital_batch_rejected(torch_cuda, wctx):
    torch = torch_cuda
    lr = full_periodic(8)
    reg = Region(wctx, lr)
    psi = torch.rand(lr.ncoeff, dtype=torch.float64, device="cuda")
    hpsi, pot = torch.zeros_like(psi), torch.zeros(lr.nisf, dtype=torch.float64, device="cuda")
    e = torch.empty(2, 1, dtype=torch.float64, device="cuda")
    first = OrbitalBatch(wctx, [(reg, psi, hpsi, pot, None)])
    second = OrbitalBatch(wctx, [(reg, psi, hpsi, pot, None)])
    with pytest.raises(WvlhError, match="code 7"):
        first.locham(e[0], e[1])
    second.locham(e[0], e[1])
    # a locham-only batch has no densities to accumulate into
    with pytest.raises(WvlhError):
        second.locden(torch.ones(1, dtype=torch.float64, device="cuda"))
    torch.cuda.synchronize()
    assert torch.isfinite(e).all()


def _serve_alone_and_mixed(torch, precision):
    specs = small_clients()
    srv = Server(precision=precision, hbm_budget=8e9, n_slots=2, scratch_per_slot=2e9)
    data = [client_data(lr, n, 100 + i) for i, (lr, n) in enumerate(specs)]
    cl = [srv.register(lr, n, psi=psi, pot=pot) for (lr, n), (psi, pot) in zip(specs, data)]
    alone = []
    for c in cl:
        rh = srv.submit(c, "H")
        srv.drain()
        rr = srv.submit(c, "rho")
        srv.drain()
        alone.append((c.hpsi.clone(), c.rho.clone(), rh.ekin, rh.epot))
    for c in cl:
        c.hpsi.zero_()
        c.rho.fill_(7.0)
    torch.cuda.synchronize()   # the slots' streams must see these writes
    n0 = srv.launches
    reqs = [srv.submit(c, k) for c in cl for k in ("H", "rho")]
    srv.drain()
    torch.cuda.synchronize()
    assert all(r.t_done is not None for r in reqs)
    # all ten requests went out in at most two launches (one per slot)
    assert srv.launches - n0 <= 2
    out = []
    for c, (hp, rho, ek, ep) in zip(cl, alone):
        rh = [r for r in reqs if r.client is c and r.kind == "H"][0]
        out.append((rel(c.hpsi.cpu(), hp.cpu()), rel(c.rho.cpu(), rho.cpu()), ek, rh.ekin, ep, rh.epot))
    return srv, cl, data, out


def test_same_alone_and_in_the_mix_fp64(oracle, torch_cuda):
    torch = torch_cuda
    srv, cl, data, out = _serve_alone_and_mixed(torch, 64)
    for dh, dr, ek, ek2, ep, ep2 in out:
        assert dh < 1e-13 and dr < 1e-13
        assert abs(ek - ek2) <= 1e-12 * abs(ek) and abs(ep - ep2) <= 1e-12 * max(abs(ep), 1.0)
    # and both agree with the oracle (client 1: free BC)
    c = cl[1]
    lr = c.locreg
    d = oracle.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
    psi, pot = data[1]
    hp = c.hpsi.cpu().numpy()
    rho_ref = np.zeros(lr.nisf)
    vol = np.prod([0.5 * h for h in lr.hgrid])
    for o in range(c.norb):
        hc, hf, _, _ = oracle.locham(d, lr.hgrid, psi[o, :lr.nvctr_c], psi[o, lr.nvctr_c:], pot)
        assert rel(hp[o], np.concatenate([hc, hf])) < 1e-13
        rho_ref = oracle.locden(d, psi[o, :lr.nvctr_c], psi[o, lr.nvctr_c:], 2.0 / vol, rho_ref)
    assert rel(c.rho.cpu().numpy(), rho_ref) < 1e-13
    srv.close()


def test_same_alone_and_in_the_mix_fp32(torch_cuda):
    torch = torch_cuda
    srv, _, _, out = _serve_alone_and_mixed(torch, 32)
    for dh, dr, ek, ek2, ep, ep2 in out:
        assert dh < 1e-6 and dr < 1e-6
        assert abs(ek - ek2) <= 1e-6 and abs(ep - ep2) <= 1e-6
    srv.close()


def test_admission_by_hbm_budget(torch_cuda):
    torch = torch_cuda
    specs = small_clients()[:3]
    from wvlh.serve import client_bytes
    need = [client_bytes(lr, n, 8) for lr, n in specs]
    scratch = 1 << 30
    srv = Server(precision=64, hbm_budget=scratch + need[0] + need[1] + 1, n_slots=1, scratch_per_slot=scratch)
    cl = [srv.register(lr, n, seed=i) for i, (lr, n) in enumerate(specs)]
    assert cl[0].admitted and cl[1].admitted and not cl[2].admitted
    r2 = srv.submit(cl[2], "H")
    r0 = srv.submit(cl[0], "rho")
    srv.drain()
    assert r0.t_done is not None and r2.t_done is None   # client 2 is not resident yet
    srv.release(cl[0])
    assert cl[2].admitted and srv.resident <= srv.capacity
    srv.drain()
    assert r2.t_done is not None and np.isfinite(r2.ekin)
    srv.close()


def test_launch_orbital_cap(torch_cuda):
    """A client with more orbitals than a launch holds is refused; with
    max_orbitals at the largest client every launch stays within the slots'
    buffers and the requests complete."""
    from wvlh.serve import AdmissionError
    specs = small_clients()
    big = max(n for _, n in specs)
    srv = Server(precision=32, hbm_budget=8e9, n_slots=2, scratch_per_slot=2e9, max_orbitals=big - 1)
    lr, n = next((lr, n) for lr, n in specs if n == big)
    with pytest.raises(AdmissionError, match="orbitals"):
        srv.register(lr, n)
    srv.close()
    srv = Server(precision=32, hbm_budget=8e9, n_slots=2, scratch_per_slot=2e9, max_orbitals=big)
    cl = [srv.register(lr, n, seed=i) for i, (lr, n) in enumerate(specs)]
    reqs = srv.replay(poisson_arrivals(5e4, 40, len(cl), seed=5))
    assert all(r.t_done is not None for r in reqs)
    assert all(np.isfinite(r.ekin) for r in reqs if r.kind == "H")
    srv.close()


def test_poisson_replay_completes(torch_cuda):
    specs = small_clients()
    srv = Server(precision=32, hbm_budget=8e9, n_slots=2, scratch_per_slot=2e9)
    cl = [srv.register(lr, n, seed=i) for i, (lr, n) in enumerate(specs)]
    reqs = srv.replay(poisson_arrivals(5e4, 60, len(cl), seed=3))
    st = latency_stats(reqs)
    assert st["n"] == 60 and 0 < st["p50_ms"] <= st["p99_ms"]
    assert 0 <= st["queued_p50_ms"] <= st["queued_p99_ms"] and 0 < st["launched_p50_ms"] <= st["launched_p99_ms"]
    assert st["tail"]["requests"] >= 1 and st["tail"]["orbitals_mean"] > 0
    assert srv.launches < 60   # requests were batched
    srv.close()


@pytest.mark.parametrize("precision,binary", [(64, True), (32, False)])
def test_evict_to_restart_files_and_restore(torch_cuda, tmp_path, precision, binary):
    """A client's orbitals leave the device as the reference's restart files
    and come back: the same H psi and energies afterwards (bit for bit with
    the binary form; FP32 values also survive the plain form's 12/10 digits)."""
    torch = torch_cuda
    specs = small_clients()[:2]
    srv = Server(precision=precision, hbm_budget=8e9, n_slots=1, scratch_per_slot=2e9)
    data = [client_data(lr, n, 300 + i) for i, (lr, n) in enumerate(specs)]
    cl = [srv.register(lr, n, psi=psi, pot=pot) for (lr, n), (psi, pot) in zip(specs, data)]
    r = srv.submit(cl[0], "H")
    srv.drain()
    before = (cl[0].hpsi.clone(), r.ekin, r.epot, cl[0].psi.clone())
    srv.evict(cl[0], str(tmp_path / "wavefunction"), binary=binary)
    assert not cl[0].admitted and cl[0].psi is None
    assert (tmp_path / ("wavefunction-k001-NR.%sb000001" % ("bin." if binary else ""))).exists()
    srv.restore(cl[0])
    assert cl[0].admitted and torch.equal(cl[0].psi, before[3])
    r = srv.submit(cl[0], "H")
    srv.drain()
    torch.cuda.synchronize()
    assert torch.equal(cl[0].hpsi, before[0]) and r.ekin == before[1] and r.epot == before[2]
    srv.close()
