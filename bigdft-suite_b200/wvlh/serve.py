"""Serving loop: H psi and density requests from many independent SCF clients.

A client is one SCF run (the reference runs one per process and calls
``local_hamiltonian_OCL`` / ``local_partial_density_OCL`` of
``bigdft/src/OpenCL/interface_ocl.f90:391-587,908-1018`` on its own queue).
Here many clients share one GPU:

* **Residency.**  A registered client's region (keys validated and decoded
  once, :class:`wvlh.batch.Region`), coefficients psi, output hpsi, ISF
  potential and FP64 density stay on the device while it is admitted.
* **Admission by HBM budget.**  A client is admitted when its resident bytes
  plus those already admitted plus the scratch reserved for the device slots
  fit the budget; otherwise it waits (FIFO) until a client leaves.
* **Continuous batching.**  Requests (``"H"``: hpsi = H psi and the energies;
  ``"rho"``: rho = sum_o hfac_o |psi_o|^2) wait in one FIFO.  Whenever one of
  the device slots (a library context with its own CUDA stream) is free, the
  waiting requests that fit its scratch share are packed into one orbital
  batch per kind (all orbitals of all picked clients in one fused launch
  sequence) and launched; requests that arrive meanwhile go to the next free
  slot, so launches of different slots overlap on the device.
* **Ordering.**  A client has at most one request of each kind in flight
  (both write the same hpsi or rho); its later requests of that kind wait.

Latency of a request = time its completion is observed on the host minus its
arrival time (both ``time.perf_counter``).
"""
import ctypes as C
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from ._lib import OrbitalDesc, WvlhError, check, lib, require_cuda
from .batch import Context, Region


class AdmissionError(WvlhError):
    pass


@dataclass(eq=False)
class Request:
    client: "Client"
    kind: str            # "H" or "rho"
    t_arrival: float
    t_launch: float = None
    t_done: float = None
    slot: int = None
    ekin: float = None   # sum_o occ_o <psi_o|T|psi_o> (H requests)
    epot: float = None   # sum_o occ_o <psi_o|V|psi_o>

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_arrival

    @property
    def scratch(self):
        return self.client.scratch_bytes


@dataclass(eq=False)
class Client:
    id: int
    locreg: object
    norb: int
    occ: np.ndarray
    region: Region = None
    psi: object = None    # (norb, ncoeff) device tensor
    hpsi: object = None
    pot: object = None    # (nisf,) device tensor
    rho: object = None    # (nisf,) float64 device tensor
    resident_bytes: int = 0
    scratch_bytes: int = 0
    admitted: bool = False
    requests_done: int = 0
    coarse_cells: int = 0
    waiting: list = field(default_factory=list)


def client_bytes(locreg, norb, elem):
    """Resident device bytes of a client: psi, hpsi, potential, FP64 density."""
    return 2 * norb * locreg.ncoeff * elem + locreg.nisf * (elem + 8)


def request_scratch(locreg, norb, elem):
    """Fused-kernel scratch bytes of one request of a client (P, Q, Z per
    orbital; the library's wvlh_region_scratch_bytes)."""
    F, I = locreg.fine, locreg.isf
    G3 = 2 * locreg.n[2]
    return norb * elem * (2 * G3 * F[1] * F[0] + G3 * I[1] * I[0])


def form_launch(waiting, busy, scratch_cap, max_orbitals):
    """Pick the requests of one launch from the FIFO `waiting`: first fit in
    arrival order, skipping requests whose (client, kind) is in flight
    (`busy`) or already picked, while the scratch of each kind's batch stays
    within scratch_cap and the orbitals within max_orbitals.  The oldest
    eligible request is always taken.  Returns {"H": [...], "rho": [...]}."""
    picked = {"H": [], "rho": []}
    used = {"H": 0, "rho": 0}
    norb = {"H": 0, "rho": 0}
    taken = set()
    for r in waiting:
        key = (r.client.id, r.kind)
        if key in busy or key in taken:
            continue
        k = r.kind
        if picked[k] and (used[k] + r.scratch > scratch_cap or norb[k] + r.client.norb > max_orbitals):
            continue
        picked[k].append(r)
        used[k] += r.scratch
        norb[k] += r.client.norb
        taken.add(key)
    return picked


class _Slot:
    """One device slot: a library context on its own stream, with the
    per-launch energy and density-weight buffers it reuses."""

    def __init__(self, index, device, max_orbitals):
        torch = require_cuda()
        self.index = index
        self.stream = torch.cuda.Stream(device)
        self.ctx = Context(device, self.stream)
        self.event = torch.cuda.Event()
        self.e_dev = torch.empty(2, max_orbitals, dtype=torch.float64, device=device)
        self.e_host = torch.empty(2, max_orbitals, dtype=torch.float64).pin_memory()
        self.hfac_dev = torch.empty(max_orbitals, dtype=torch.float64, device=device)
        self.hfac_host = torch.empty(max_orbitals, dtype=torch.float64).pin_memory()
        self.requests = None


class Server:
    """Continuous-batching server of H psi and density requests on one GPU.

    precision: 32 (FP32 convolutions, FP64 energies and densities) or 64.
    hbm_budget: bytes of device memory the server may use for resident
    client state plus the slots' scratch (scratch_per_slot each)."""

    def __init__(self, device=0, precision=32, hbm_budget=150e9, n_slots=2, scratch_per_slot=16e9,
                 max_orbitals=4096):
        torch = require_cuda()
        self.torch = torch
        self.device = device
        self.precision = precision
        self.dtype = torch.float32 if precision == 32 else torch.float64
        self.elem = 4 if precision == 32 else 8
        self.hbm_budget = int(hbm_budget)
        self.scratch_per_slot = int(scratch_per_slot)
        self.max_orbitals = max_orbitals
        self.slots = [_Slot(i, device, max_orbitals) for i in range(n_slots)]
        self.clients = []
        self.pending = deque()        # clients waiting for admission
        self.queue = []               # waiting requests, arrival order
        self.busy = set()             # (client id, kind) in flight
        self.done = []
        self.resident = 0
        self.launches = 0
        self.kernel_launches = 0
        # the admission view of memory: budget minus the slots' scratch
        self.capacity = self.hbm_budget - n_slots * self.scratch_per_slot
        if self.capacity <= 0:
            raise WvlhError("HBM budget smaller than the slots' scratch")

    # ------------------------------------------------------------------ clients
    def register(self, locreg, norb, seed=0, psi=None, pot=None, occ=2.0):
        """Add a client; it becomes resident now if the budget allows, else it
        waits for admission.  psi: (norb, ncoeff) array (host or device) or
        None for seeded uniform(-1, 1) rows drawn on the device; pot: ISF
        potential or None for zero.  Raises AdmissionError if the client can
        never fit (its resident bytes above the capacity, one request's
        scratch above a slot's share, or more orbitals than a launch holds:
        max_orbitals sizes each slot's energy and occupation buffers)."""
        c = Client(id=len(self.clients), locreg=locreg, norb=int(norb), occ=np.full(int(norb), float(occ)))
        c.coarse_cells = locreg.coarse_cells * c.norb
        c.resident_bytes = client_bytes(locreg, c.norb, self.elem)
        c.scratch_bytes = request_scratch(locreg, c.norb, self.elem)
        if c.resident_bytes > self.capacity:
            raise AdmissionError("client %d needs %d resident bytes, capacity %d"
                                 % (c.id, c.resident_bytes, self.capacity))
        if c.norb > self.max_orbitals:
            raise AdmissionError("client %d has %d orbitals, a launch holds at most %d"
                                 % (c.id, c.norb, self.max_orbitals))
        if c.scratch_bytes > self.scratch_per_slot:
            raise AdmissionError("client %d: one request needs %d scratch bytes, a slot has %d"
                                 % (c.id, c.scratch_bytes, self.scratch_per_slot))
        c._init = (seed, psi, pot)
        self.clients.append(c)
        self.pending.append(c)
        self._admit()
        return c

    def _admit(self):
        while self.pending and self.resident + self.pending[0].resident_bytes <= self.capacity:
            c = self.pending.popleft()
            self._make_resident(c)

    def _make_resident(self, c):
        torch = self.torch
        dev = self.device
        c.region = Region(self.slots[0].ctx, c.locreg)
        seed, psi, pot = c._init
        ncoeff, nisf = c.region.psi_size, c.region.grid_size
        if psi is None:
            g = torch.Generator(device=dev)
            g.manual_seed(int(seed))
            c.psi = torch.rand(c.norb, ncoeff, generator=g, device=dev, dtype=torch.float64).mul_(2).sub_(1)
            c.psi = c.psi.to(self.dtype)
        else:
            c.psi = torch.as_tensor(psi).to(device=dev, dtype=self.dtype).reshape(c.norb, ncoeff).contiguous()
        c.hpsi = torch.zeros_like(c.psi)
        if pot is None:
            c.pot = torch.zeros(nisf, dtype=self.dtype, device=dev)
        else:
            c.pot = torch.as_tensor(pot).to(device=dev, dtype=self.dtype).reshape(nisf).contiguous()
        c.rho = torch.zeros(nisf, dtype=torch.float64, device=dev)
        vol = float(np.prod([0.5 * h for h in c.locreg.hgrid]))
        c.hfac = c.occ / vol
        # the slots' streams use these buffers: finish their initialisation first
        torch.cuda.current_stream(dev).synchronize()
        c.admitted = True
        c._init = None
        self.resident += c.resident_bytes
        for r in c.waiting:
            self.queue.append(r)
        c.waiting = []
        self.queue.sort(key=lambda r: r.t_arrival)

    def release(self, c):
        """Drop a client's device state (after its requests completed) and
        admit waiting clients in its place."""
        if any(k[0] == c.id for k in self.busy) or any(r.client is c for r in self.queue):
            raise WvlhError("client %d still has requests" % c.id)
        if c.admitted:
            c.psi = c.hpsi = c.pot = c.rho = None
            c.region.close()
            c.admitted = False
            self.resident -= c.resident_bytes
        self._admit()

    def evict(self, c, radical, binary=True):
        """Move a client's orbitals out of device memory into the reference's
        restart files (wvlh.restart, one file per orbital: <radical>-k001-NR...)
        and release its device state; its potential stays in host memory.
        Restore it with restore()."""
        from .restart import write_waves
        if not c.admitted:
            raise WvlhError("client %d is not resident" % c.id)
        if any(k[0] == c.id for k in self.busy) or any(r.client is c for r in self.queue):
            raise WvlhError("client %d still has requests" % c.id)
        write_waves(radical, c.psi.double().cpu().numpy(), c.locreg, binary=binary)
        pot = c.pot.cpu().numpy()
        self.release(c)
        c._evicted = (radical, binary, pot)

    def restore(self, c):
        """Read an evicted client's orbitals back and queue it for admission
        (admitted now if the budget allows)."""
        from .restart import read_waves
        radical, binary, pot = getattr(c, "_evicted", (None, None, None))
        if radical is None:
            raise WvlhError("client %d was not evicted" % c.id)
        psi = read_waves(radical, c.norb, c.locreg, binary=binary)
        c._init = (0, psi, pot)
        c._evicted = None
        self.pending.append(c)
        self._admit()

    # ----------------------------------------------------------------- requests
    def submit(self, c, kind, t_arrival=None):
        if kind not in ("H", "rho"):
            raise WvlhError("request kind is 'H' or 'rho'")
        r = Request(client=c, kind=kind, t_arrival=time.perf_counter() if t_arrival is None else t_arrival)
        if c.admitted:
            self.queue.append(r)
        else:
            c.waiting.append(r)
        return r

    def _table(self, reqs, kind):
        """(n, 5) uint64 rows of wvlh_orbital for all orbitals of reqs."""
        rows = []
        for r in reqs:
            c = r.client
            n = c.norb
            t = np.zeros((n, 5), np.uint64)
            t[:, 0] = c.region.h.value
            step = c.region.psi_size * self.elem
            t[:, 1] = c.psi.data_ptr() + step * np.arange(n, dtype=np.uint64)
            if kind == "H":
                t[:, 2] = c.hpsi.data_ptr() + step * np.arange(n, dtype=np.uint64)
                t[:, 3] = c.pot.data_ptr()
            else:
                t[:, 4] = c.rho.data_ptr()
            rows.append(t)
        return np.ascontiguousarray(np.concatenate(rows))

    def _batch(self, ctx, table):
        h = C.c_void_p()
        check(lib().wvlh_batch_create_orbitals(ctx.h, len(table), table.ctypes.data_as(C.POINTER(OrbitalDesc)),
                                               C.byref(h)), "wvlh_batch_create_orbitals")
        return h

    def _launch(self, slot, picked, now):
        torch = self.torch
        L = lib()
        reqs = picked["H"] + picked["rho"]
        with torch.cuda.stream(slot.stream):
            nH = sum(r.client.norb for r in picked["H"])
            if picked["H"]:
                h = self._batch(slot.ctx, self._table(picked["H"], "H"))
                try:
                    e = slot.e_dev
                    rc = L.wvlh_locham_batched(h, self.precision, None, None, None, C.c_void_p(e[0].data_ptr()),
                                               C.c_void_p(e[1].data_ptr()), 0)
                finally:
                    L.wvlh_batch_destroy(h)
                check(rc, "wvlh_locham_batched")
                slot.e_host[0, :nH].copy_(slot.e_dev[0, :nH], non_blocking=True)
                slot.e_host[1, :nH].copy_(slot.e_dev[1, :nH], non_blocking=True)
                self.kernel_launches += 4   # K1, K2, K3, energy reduction
            if picked["rho"]:
                torch._foreach_zero_([r.client.rho for r in picked["rho"]])
                hf = np.concatenate([r.client.hfac for r in picked["rho"]])
                slot.hfac_host[:len(hf)].numpy()[:] = hf
                slot.hfac_dev[:len(hf)].copy_(slot.hfac_host[:len(hf)], non_blocking=True)
                h = self._batch(slot.ctx, self._table(picked["rho"], "rho"))
                try:
                    rc = L.wvlh_locden_batched(h, self.precision, None, C.c_void_p(slot.hfac_dev.data_ptr()), None)
                finally:
                    L.wvlh_batch_destroy(h)
                check(rc, "wvlh_locden_batched")
                self.kernel_launches += 3   # K1, density, chunk reduction
            slot.event.record(slot.stream)
        for r in reqs:
            r.t_launch = now
            r.slot = slot.index
            self.busy.add((r.client.id, r.kind))
        ids = set(map(id, reqs))
        self.queue = [r for r in self.queue if id(r) not in ids]
        slot.requests = picked
        self.launches += 1

    def _complete(self, slot, now):
        picked = slot.requests
        o = 0
        eh = slot.e_host.numpy()
        for r in picked["H"]:
            n = r.client.norb
            r.ekin = float(np.dot(r.client.occ, eh[0, o:o + n]))
            r.epot = float(np.dot(r.client.occ, eh[1, o:o + n]))
            o += n
        for r in picked["H"] + picked["rho"]:
            r.t_done = now
            r.client.requests_done += 1
            self.busy.discard((r.client.id, r.kind))
            self.done.append(r)
        slot.requests = None

    def poll(self):
        """Complete finished launches, then fill every free slot."""
        now = time.perf_counter()
        for s in self.slots:
            if s.requests is not None and s.event.query():
                self._complete(s, now)
        for s in self.slots:
            if s.requests is None and self.queue:
                picked = form_launch(self.queue, self.busy, self.scratch_per_slot, self.max_orbitals)
                if picked["H"] or picked["rho"]:
                    self._launch(s, picked, time.perf_counter())

    @property
    def idle(self):
        return not self.queue and all(s.requests is None for s in self.slots)

    def drain(self):
        while not self.idle:
            self.poll()

    def replay(self, arrivals, clients=None):
        """Serve a list of (t, client index, kind) arrivals in real time,
        starting now; returns the requests (with latencies) in arrival order."""
        clients = self.clients if clients is None else clients
        t0 = time.perf_counter()
        out = []
        i = 0
        while i < len(arrivals) or not self.idle:
            now = time.perf_counter() - t0
            while i < len(arrivals) and arrivals[i][0] <= now:
                t, ci, kind = arrivals[i]
                out.append(self.submit(clients[ci], kind, t0 + t))
                i += 1
            self.poll()
        return out

    def close(self):
        self.torch.cuda.synchronize(self.device)
        for c in self.clients:
            if c.admitted:
                c.region.close()
        for s in self.slots:
            s.ctx.close()


def latency_stats(reqs):
    """p50 / p99 / mean latency (ms) of completed requests, split into the
    time queued before their launch and the time from launch to completion
    (kernels, plus any launch of the other slot ahead of them on the
    device); "tail" gives the mean of both parts and the mean orbital count
    over the requests at or above the p99 latency, against all requests."""
    done = [r for r in reqs if r.latency is not None]
    if not done:
        return {"n": 0}
    lat = np.array([r.latency for r in done]) * 1e3
    wait = np.array([r.t_launch - r.t_arrival for r in done]) * 1e3
    run = lat - wait
    norb = np.array([r.client.norb for r in done], dtype=float)
    p99 = float(np.percentile(lat, 99))
    top = lat >= p99
    return {"n": int(len(lat)), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": p99,
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
            "queued_p50_ms": float(np.percentile(wait, 50)), "queued_p99_ms": float(np.percentile(wait, 99)),
            "launched_p50_ms": float(np.percentile(run, 50)), "launched_p99_ms": float(np.percentile(run, 99)),
            "tail": {"requests": int(top.sum()), "queued_mean_ms": float(wait[top].mean()),
                     "launched_mean_ms": float(run[top].mean()), "orbitals_mean": float(norb[top].mean()),
                     "orbitals_mean_all": float(norb.mean())}}
