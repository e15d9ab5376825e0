"""Multi-process host logic of the orbital sharding (no GPU): world_size-2
gloo process groups on CPU run the same exchange code that NCCL runs on
GPUs (energy all-reduce, density all-reduce and z-slab reduce-scatter, the
overlap's orbital -> component transposition and all-reduce)."""
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from wvlh.keys import Locreg
from wvlh.shard import (allreduce_energies, component_slices, orbital_cost, overlap_sharded, reduce_density,
                        shard_orbitals, z_slabs)

GRID = (6, 5, 7)  # (I1, I2, I3) of a small ISF grid


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_data(rank, norb=5):
    g = torch.Generator().manual_seed(100 + rank)
    ekin = torch.rand(norb, generator=g, dtype=torch.float64) * 50
    epot = -torch.rand(norb, generator=g, dtype=torch.float64) * 10
    rho = torch.rand(GRID[0] * GRID[1] * GRID[2], generator=g, dtype=torch.float64)
    return ekin, epot, rho


def _worker(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        ekin, epot, rho = _rank_data(rank)
        occ = torch.full_like(ekin, 2.0)
        ek, ep = allreduce_energies(ekin, epot, occ)
        slab = reduce_density(rho.clone(), GRID, scatter=True)
        full = reduce_density(rho.clone(), GRID, scatter=False)
        out[rank] = (ek, ep, slab.numpy().copy(), full.numpy().copy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_energy_and_density_exchanges(world):
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    data = [_rank_data(r) for r in range(world)]
    ek_ref = sum(2.0 * d[0].sum().item() for d in data)
    ep_ref = sum(2.0 * d[1].sum().item() for d in data)
    rho_ref = sum(d[2] for d in data).numpy()
    slabs = z_slabs(GRID[2], world)
    plane = GRID[0] * GRID[1]
    for r in range(world):
        ek, ep, slab, full = out[r]
        assert abs(ek - ek_ref) <= 1e-12 * abs(ek_ref) and abs(ep - ep_ref) <= 1e-12 * abs(ep_ref)
        assert np.allclose(full, rho_ref, rtol=1e-15, atol=0)
        a, b = slabs[r]
        assert np.allclose(slab, rho_ref[a * plane:b * plane], rtol=1e-15, atol=0)


def test_shard_orbitals_contiguous_and_balanced():
    rng = np.random.default_rng(0)
    costs = rng.integers(1000, 5000, 257)
    for world in (1, 2, 3, 8):
        parts = shard_orbitals(costs, world)
        assert parts[0][0] == 0 and parts[-1][1] == len(costs)
        assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
        loads = [costs[a:b].sum() for a, b in parts]
        assert max(loads) - costs.sum() / world <= costs.max()
    assert shard_orbitals([5, 5], 4)[-1] == (2, 2)   # more ranks than orbitals: empty ranges


def test_z_slabs_and_cost():
    assert z_slabs(7, 3) == [(0, 3), (3, 5), (5, 7)]
    m = np.ones((4, 4, 4), bool)
    f = np.zeros((4, 4, 4), bool)
    f[1:3, 1:3, 1:3] = True
    lr = Locreg.from_masks(m, f, (0, 0, 0), (0.5, 0.5, 0.5))
    assert orbital_cost(lr) == 64 + 7 * 8


OV_COUNTS = {2: [5, 3], 3: [4, 0, 6]}   # orbitals per rank (one rank may hold none)
OV_K = 29                               # coefficients (not a multiple of the ranks)


def _ov_psi(world):
    g = torch.Generator().manual_seed(7)
    return torch.rand(sum(OV_COUNTS[world]), OV_K, generator=g, dtype=torch.float64) * 2 - 1


def _ov_worker(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        psi = _ov_psi(world)
        c = OV_COUNTS[world]
        mine = psi[sum(c[:rank]):sum(c[:rank + 1])].clone()
        S = overlap_sharded(mine, gram=lambda X: X @ X.T)
        out[rank] = S.numpy().copy()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_overlap_transposition_and_allreduce(world):
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_ov_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    psi = _ov_psi(world).numpy()
    ref = psi @ psi.T
    for r in range(world):
        assert np.abs(out[r] - ref).max() <= 1e-13 * np.abs(ref).max()
    assert component_slices(OV_K, world)[-1][1] == OV_K
