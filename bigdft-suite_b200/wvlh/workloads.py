"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset exists for this path; inputs are synthetic:

* periodic boxes with every coarse cell carrying 1 scaling + 7 wavelet
  coefficients (the full mask), coefficients uniform(-1, 1);
* free-BC localisation regions with all coarse cells occupied and a fine
  region that is an ellipsoid of radius 0.4 x the box per axis;
* a local potential that is a sum of 4 Gaussians (centres uniform in the box,
  widths uniform in [1, 3] bohr, depths uniform in [-2, -0.5] Ha), evaluated
  on the ISF grid with the periodic minimum image where the box is periodic.
"""
import numpy as np

from .keys import Locreg


def full_periodic(n, hgrid=0.45):
    N = (n, n, n) if np.isscalar(n) else tuple(n)
    mask = np.ones(N[::-1], bool)
    return Locreg.from_masks(mask, mask, (1, 1, 1), (hgrid,) * 3)


def free_sphere(N, hgrid=0.45, radius_frac=0.4):
    """All coarse cells occupied, fine region an ellipsoid centred in the box."""
    N = tuple(int(v) for v in N)
    mask_c = np.ones(N[::-1], bool)
    idx = np.meshgrid(*[np.arange(v) for v in N[::-1]], indexing="ij")  # (i3, i2, i1)
    r2 = np.zeros(N[::-1])
    for ax, n in zip(idx, N[::-1]):
        c = (n - 1) / 2.0
        r2 += ((ax - c) / (radius_frac * n)) ** 2
    mask_f = r2 <= 1.0
    return Locreg.from_masks(mask_c, mask_f, (0, 0, 0), (hgrid,) * 3)


def _gaussian_factors(lr, rng, ngauss):
    """Depth and the three 1D factors of each Gaussian of the potential."""
    hf = [0.5 * h for h in lr.hgrid]
    I = lr.isf
    coords = []
    for d in range(3):
        off = 0 if lr.periodic[d] else -14       # ISF index r <-> fine position r-14 (free)
        coords.append((np.arange(I[d]) + off) * hf[d])
    L = [lr.n[d] * lr.hgrid[d] for d in range(3)]
    out = []
    for _ in range(ngauss):
        cen = [rng.uniform(0, L[d]) for d in range(3)]
        w = rng.uniform(1.0, 3.0)
        dep = rng.uniform(-2.0, -0.5)
        e = []
        for d in range(3):   # the Gaussian is separable: product of 1D factors
            dx = coords[d] - cen[d]
            if lr.periodic[d]:
                dx = dx - L[d] * np.round(dx / L[d])
            e.append(np.exp(-dx ** 2 / (2 * w * w)))
        out.append((dep, e))
    return out


def gaussian_potential(lr, rng, ngauss=4):
    """V on the ISF grid of lr, flattened x-fastest (float64)."""
    I = lr.isf
    V = np.zeros((I[2], I[1], I[0]))
    for dep, e in _gaussian_factors(lr, rng, ngauss):
        V += dep * e[2][:, None, None] * e[1][None, :, None] * e[0][None, None, :]
    return V.ravel()


def gaussian_potential_device(lr, rng, device, ngauss=4):
    """The same potential (same draws from rng) evaluated on the device (torch float64)."""
    import torch
    I = lr.isf
    V = torch.zeros(I[2], I[1], I[0], dtype=torch.float64, device=device)
    for dep, e in _gaussian_factors(lr, rng, ngauss):
        ex, ey, ez = (torch.tensor(v, device=device) for v in e)
        V += dep * ez[:, None, None] * ey[None, :, None] * ex[None, None, :]
    return V.reshape(-1)


def random_psi(lr, norb, rng, normalize=False):
    psi = rng.uniform(-1.0, 1.0, (norb, lr.ncoeff))
    if normalize:
        psi /= np.linalg.norm(psi, axis=1, keepdims=True)
    return psi


def batched_periodic(n=48, norb=256, seed=1, hgrid=0.45):
    """Config of the batched benchmark: norb normalised orbitals on one n^3 periodic box."""
    rng = np.random.default_rng(seed)
    lr = full_periodic(n, hgrid)
    psi = random_psi(lr, norb, rng, normalize=True)
    pot = gaussian_potential(lr, rng)
    return lr, psi, pot


def single_orbital(n=32, seed=0, hgrid=0.45):
    """One orbital of uniform(-1, 1) coefficients on a periodic n^3 box with
    the 4-Gaussian potential (the single-orbital plain FP64 workload)."""
    rng = np.random.default_rng(seed)
    lr = full_periodic(n, hgrid)
    psi = random_psi(lr, 1, rng)[0]
    pot = gaussian_potential(lr, rng)
    return lr, psi, pot


def batched_periodic_device(torch, device, n=48, norb=256, seed=1000, pot_seed=1234, hgrid=0.45):
    """The batched workload generated on the device: norb orbitals of
    uniform(-1, 1) coefficients from a torch generator seeded with `seed`,
    each normalised, packed back to back (float64, flat), and the 4-Gaussian
    potential drawn from numpy's generator seeded with `pot_seed`."""
    lr = full_periodic(n, hgrid)
    pot = torch.tensor(gaussian_potential(lr, np.random.default_rng(pot_seed)), device=device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    psi = torch.rand(norb, lr.ncoeff, generator=g, device=device, dtype=torch.float64) * 2 - 1
    psi /= psi.norm(dim=1, keepdim=True)
    return lr, psi.reshape(-1).contiguous(), pot


def free_regions(nlr=1024, nmin=20, nmax=40, seed=2, hgrid=0.45):
    """nlr free-BC regions of uneven size, one support function each, one potential each."""
    rng = np.random.default_rng(seed)
    lrs, psis, pots = [], [], []
    for _ in range(nlr):
        N = tuple(int(v) for v in rng.integers(nmin, nmax + 1, 3))
        lr = free_sphere(N, hgrid)
        lrs.append(lr)
        psis.append(random_psi(lr, 1, rng, normalize=True)[0])
        pots.append(gaussian_potential(lr, rng))
    return lrs, psis, pots


def serving_clients(nclient=64, nmin=16, nmax=64, omin=4, omax=128, p_periodic=0.5, seed=4, hgrid=0.45):
    """Clients of the serving benchmark: each an independent SCF run with its
    own box (coarse cells per dimension uniform in [nmin, nmax]), periodic
    (every cell fine) or free (fine ellipsoid) with probability p_periodic,
    and uniform [omin, omax] orbitals.  Returns (locreg, norb, seed) per
    client; coefficients and potentials are drawn from the per-client seed
    where they are needed (on the device, see wvlh.serve)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nclient):
        N = tuple(int(v) for v in rng.integers(nmin, nmax + 1, 3))
        periodic = rng.uniform() < p_periodic
        lr = full_periodic(N, hgrid) if periodic else free_sphere(N, hgrid)
        norb = int(rng.integers(omin, omax + 1))
        out.append((lr, norb, int(rng.integers(1 << 30))))
    return out


def poisson_arrivals(rate, nreq, nclient, seed=5, p_density=0.5):
    """nreq requests at Poisson times of mean rate `rate` (1/s), each from a
    uniform client, a density request with probability p_density (else H psi).
    Returns a list of (t, client, kind) sorted by t, kind in {"H", "rho"}."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, nreq))
    cl = rng.integers(0, nclient, nreq)
    kind = rng.uniform(size=nreq) < p_density
    return [(float(t[i]), int(cl[i]), "rho" if kind[i] else "H") for i in range(nreq)]
