"""Orbital sharding over GPUs (one process per GPU) and the two exchanges the
path has: energies and densities.

The reference distributes orbitals over MPI ranks (``orbs%norbp`` /
``orbs%isorb``, the per-rank loop of ``LocalHamiltonianApplication``,
``bigdft/src/hpsiortho.f90:934-958``); H psi of an orbital needs nothing from
other ranks.  The exchanges are:

* energies: a sum over ranks of a few doubles (``fmpi_allreduce`` of the
  energy terms, ``hpsiortho.f90:1572``) -> :func:`allreduce_energies`;
* density: each rank's partial rho of its orbitals, summed over ranks and
  either replicated (all-reduce) or left distributed in z-slabs
  (``MPI_REDUCE_SCATTER`` in ``communicate_density``, ``sumrho.f90:219``)
  -> :func:`reduce_density`;
* overlap S = Psi Psi^T of orbitals held by different ranks: the orbital ->
  component transposition (``transpose_v``, ``communications.f90:2318``, an
  all-to-all), the symmetric product over the rank's slice of components
  (``getOverlap``, ``wfn_opt/orthogonality.f90:2624-2697``) and the sum of the
  partial matrices over ranks (``:2695``) -> :func:`overlap_sharded`.

These functions take torch tensors and a ``torch.distributed`` process group:
NCCL on GPUs, gloo for the CPU tests of this logic.
"""
import numpy as np


def orbital_cost(locreg):
    """Relative cost of one orbital of a region: coarse cells plus the fine
    cells weighted by the seven wavelet components they carry."""
    return locreg.nvctr_c + 7 * locreg.nvctr_f


def shard_orbitals(costs, world_size):
    """Split orbitals (in order) into world_size contiguous ranges of nearly
    equal total cost, like the reference's contiguous orbs%isorb ranges.
    Returns the (start, stop) range of each rank."""
    costs = np.asarray(costs, np.float64)
    n = len(costs)
    if world_size <= 0:
        raise ValueError("world_size must be positive")
    cum = np.concatenate([[0.0], np.cumsum(costs)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world_size):
        # first index whose prefix reaches r/world of the total, kept monotone
        b = int(np.searchsorted(cum, total * r / world_size, side="left"))
        b = min(max(b, bounds[-1]), n)
        bounds.append(b)
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world_size)]


def allreduce_energies(ekin, epot, occ, group=None):
    """Global E_kin and E_pot: occupation-weighted sums of this rank's
    per-orbital energies, summed over ranks (FP64).  ekin/epot/occ: tensors
    of this rank's orbitals (on the process group's device)."""
    import torch
    import torch.distributed as dist
    e = torch.stack([(occ * ekin).sum(), (occ * epot).sum()]).to(torch.float64)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(e, group=group)
    return float(e[0]), float(e[1])


def z_slabs(n3, world_size):
    """z-planes [start, stop) of each rank's slab of an n3-plane grid (the
    first n3 % world_size ranks take one plane more)."""
    base, extra = divmod(n3, world_size)
    out, s = [], 0
    for r in range(world_size):
        k = base + (1 if r < extra else 0)
        out.append((s, s + k))
        s += k
    return out


def reduce_density(rho, grid, group=None, scatter=False):
    """Sum the ranks' partial densities rho (FP64, ISF grid `grid` = (I1, I2,
    I3), x fastest).  scatter=False: every rank gets the full sum (in place).
    scatter=True: returns this rank's z-slab (planes of z_slabs) of the sum."""
    import torch
    import torch.distributed as dist
    I1, I2, I3 = grid
    if rho.numel() != I1 * I2 * I3 or rho.dtype != torch.float64:
        raise ValueError("rho must be the float64 ISF grid")
    ws = dist.get_world_size(group) if dist.is_initialized() else 1
    if not scatter:
        if ws > 1:
            dist.all_reduce(rho, group=group)
        return rho
    slabs = z_slabs(I3, ws)
    rank = dist.get_rank(group) if ws > 1 else 0
    plane = I1 * I2
    if ws == 1:
        return rho.view(I3, plane)[slabs[0][0]:slabs[0][1]].reshape(-1)
    # reduce-scatter wants equal chunks: pad every slab to the largest
    m = max(b - a for a, b in slabs)
    src = torch.zeros(ws, m * plane, dtype=rho.dtype, device=rho.device)
    v = rho.view(I3, plane)
    for r, (a, b) in enumerate(slabs):
        src[r, :(b - a) * plane] = v[a:b].reshape(-1)
    out = torch.empty(m * plane, dtype=rho.dtype, device=rho.device)
    dist.reduce_scatter_tensor(out, src.reshape(-1), group=group)
    a, b = slabs[rank]
    return out[:(b - a) * plane]


def component_slices(ncoeff, world_size):
    """[start, stop) of each rank's slice of the coefficients in the component
    distribution (the first ncoeff % world_size ranks take one more)."""
    return z_slabs(ncoeff, world_size)


def overlap_sharded(psi_local, group=None, gram=None, ctx=None):
    """S = Psi Psi^T (FP64, norb x norb on every rank) for orbitals sharded
    over the ranks in order (rank r holds the (norb_r, ncoeff) rows
    psi_local, ranks in orbital order).  The rows are transposed to the
    component distribution with one all-to-all (each rank then holds all
    orbitals on its slice of components), the slice's Gram matrix is formed
    locally and the partial matrices are summed with an all-reduce.  gram(X)
    returns X X^T: by default the library's FP64 tensor-core overlap kernel
    (wvlh_overlap, needs ctx) for device tensors; the CPU tests pass a
    matrix product."""
    import torch
    import torch.distributed as dist
    if psi_local.dim() != 2:
        raise ValueError("psi_local must be (norb_local, ncoeff)")
    if gram is None:
        if ctx is None:
            raise ValueError("the device overlap needs the context (ctx)")
        from .ortho import overlap as _overlap

        def gram(X):
            return _overlap(ctx, X)
    ws = dist.get_world_size(group) if dist.is_initialized() else 1
    if ws == 1:
        return gram(psi_local.contiguous())
    rank = dist.get_rank(group)
    nloc, K = psi_local.shape
    counts = torch.zeros(ws, dtype=torch.int64, device=psi_local.device)
    counts[rank] = nloc
    dist.all_reduce(counts, group=group)
    counts = [int(c) for c in counts.tolist()]
    norb = sum(counts)
    sl = component_slices(K, ws)
    lens = [b - a for a, b in sl]
    # orbital -> component distribution: rank s receives every rank's rows
    # restricted to its slice s (packed contiguous per destination)
    send = torch.cat([psi_local[:, a:b].reshape(-1) for a, b in sl]) if nloc else \
        psi_local.new_empty(0)
    recv = psi_local.new_empty(norb * lens[rank])
    dist.all_to_all_single(recv, send, output_split_sizes=[c * lens[rank] for c in counts],
                           input_split_sizes=[nloc * n for n in lens], group=group)
    X = recv.view(norb, lens[rank])       # ranks in orbital order
    S = gram(X) if lens[rank] else torch.zeros(norb, norb, dtype=torch.float64, device=psi_local.device)
    S = S.to(torch.float64).contiguous()
    dist.all_reduce(S, group=group)
    return S


class RankFailure(RuntimeError):
    """Raised on the surviving ranks when a peer did not reach a step."""

    def __init__(self, step, missing):
        super().__init__("step %d: rank(s) %s did not arrive" % (step, ", ".join(map(str, missing))))
        self.step = step
        self.missing = list(missing)


class StepMonitor:
    """Host-side failure detection between steps, before any collective of
    the step is entered: each rank records in a key-value store (a
    torch.distributed TCPStore) that it reached step k, then waits at most
    `timeout` seconds for the others.  A rank that left between steps (an
    exception, a crash) is found here and reported with RankFailure, so no
    rank starts a collective (or a kernel that would wait for a peer) that
    the missing rank will never join.  A collective already in flight when a
    rank dies is ended by the process group's own timeout instead."""

    def __init__(self, store, rank, world, prefix="wvlh/step"):
        self.store, self.rank, self.world, self.prefix = store, rank, world, prefix

    def _key(self, step, r):
        return "%s/%d/%d" % (self.prefix, step, r)

    def arrive(self, step):
        self.store.set(self._key(step, self.rank), "1")

    def missing(self, step, timeout=2.0, poll=0.02):
        import time
        keys = [self._key(step, r) for r in range(self.world)]
        t0 = time.monotonic()
        while True:
            absent = [r for r, k in enumerate(keys) if not self.store.check([k])]
            if not absent or time.monotonic() - t0 > timeout:
                return absent
            time.sleep(poll)

    def barrier(self, step, timeout=2.0):
        """arrive at step, then raise RankFailure if a peer does not"""
        self.arrive(step)
        absent = self.missing(step, timeout)
        if absent:
            raise RankFailure(step, absent)
