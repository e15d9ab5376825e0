"""GPU parity of the compressed scalar products (the reference's wpdot,
wavelib/scalprod.f90:3222) against the oracle's restatement of its loop:
FP64 within 1e-13 of the largest product magnitude; FP32 rows are widened
(products exact in FP64), same bar."""
import numpy as np
import pytest

from wvlh._lib import WvlhError
from wvlh.batch import Region, scalar_products
from wvlh.keys import Locreg

pytestmark = pytest.mark.gpu


def region(rng, N, pc, pf):
    m = rng.random(N[::-1]) < pc
    f = m & (rng.random(N[::-1]) < pf)
    return Locreg.from_masks(m, f, (0, 0, 0), (0.45, 0.45, 0.45))


def keys(lr):
    return (lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)


@pytest.mark.parametrize("seed,dtype_name", [(0, "float64"), (1, "float64"), (2, "float32"), (3, "float64")])
def test_wpdot_matches_oracle(oracle, torch_cuda, wctx, seed, dtype_name):
    torch = torch_cuda
    rng = np.random.default_rng(seed)
    N = tuple(int(v) for v in rng.integers(8, 20, 3))
    la = region(rng, N, rng.uniform(0.4, 0.9), 0.5)
    lb = region(rng, N, rng.uniform(0.2, 0.7), 0.0 if seed == 3 else 0.4)   # seed 3: b without fine part
    na, nb = 3, 5
    A = rng.uniform(-1, 1, (na, la.ncoeff + 7))    # row stride above the vector length
    B = rng.uniform(-1, 1, (nb, lb.ncoeff))
    dt = getattr(torch, dtype_name)
    if dtype_name == "float32":
        A, B = A.astype(np.float32).astype(np.float64), B.astype(np.float32).astype(np.float64)
    ta = torch.tensor(A, dtype=dt, device="cuda")[:, :la.ncoeff]
    tb = torch.tensor(B, dtype=dt, device="cuda")
    got = scalar_products(wctx, Region(wctx, la), ta, Region(wctx, lb), tb).cpu().numpy()
    ref = np.array([[oracle.wpdot(keys(la), A[i, :la.ncoeff], keys(lb), B[j]) for j in range(nb)]
                    for i in range(na)])
    assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
    # deterministic: a second call gives the same bits
    again = scalar_products(wctx, Region(wctx, la), ta, Region(wctx, lb), tb).cpu().numpy()
    assert np.array_equal(got, again)


def test_wpdot_self_is_squared_norm(torch_cuda, wctx):
    torch = torch_cuda
    rng = np.random.default_rng(5)
    lr = region(rng, (12, 11, 10), 0.6, 0.5)
    v = torch.tensor(rng.uniform(-1, 1, (2, lr.ncoeff)), device="cuda")
    r = Region(wctx, lr)
    s = scalar_products(wctx, r, v, r, v).cpu().numpy()
    vv = v.cpu().numpy()
    assert np.allclose(np.diag(s), (vv * vv).sum(axis=1), rtol=1e-14, atol=0)


def test_wpdot_rejects_different_boxes(torch_cuda, wctx):
    torch = torch_cuda
    rng = np.random.default_rng(6)
    la, lb = region(rng, (8, 8, 8), 0.5, 0.5), region(rng, (9, 8, 8), 0.5, 0.5)
    a = torch.zeros(1, la.ncoeff, dtype=torch.float64, device="cuda")
    b = torch.zeros(1, lb.ncoeff, dtype=torch.float64, device="cuda")
    with pytest.raises(WvlhError):
        scalar_products(wctx, Region(wctx, la), a, Region(wctx, lb), b)
