"""GPU parity of the FP64 tensor-core overlap S = Psi Psi^T (getOverlap,
wfn_opt/orthogonality.f90:2624-2697) against the oracle's syrk restatement,
and of the Cholesky / Loewdin orthonormalisation built on it."""
import numpy as np
import pytest

from wvlh.ortho import orthonormalize, overlap

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("norb,K", [(7, 1000), (64, 4096), (100, 12345), (256, 30000)])
def test_overlap_matches_oracle(oracle, torch_cuda, wctx, norb, K):
    torch = torch_cuda
    rng = np.random.default_rng(norb + K)
    psi = rng.uniform(-1, 1, (norb, K))
    S = overlap(wctx, torch.tensor(psi, device="cuda")).cpu().numpy()
    ref = oracle.overlap(psi)
    assert np.abs(S - ref).max() / np.abs(ref).max() < 1e-13
    assert np.array_equal(S, S.T)


def test_overlap_fp32_rows_widened(oracle, torch_cuda, wctx):
    torch = torch_cuda
    rng = np.random.default_rng(1)
    psi32 = rng.uniform(-1, 1, (40, 5000)).astype(np.float32)
    S = overlap(wctx, torch.tensor(psi32, device="cuda")).cpu().numpy()
    ref = oracle.overlap(psi32.astype(np.float64))
    assert np.abs(S - ref).max() / np.abs(ref).max() < 1e-13


def test_overlap_row_stride_and_batch_layout(oracle, torch_cuda, wctx):
    torch = torch_cuda
    rng = np.random.default_rng(2)
    full = rng.uniform(-1, 1, (12, 3000))
    t = torch.tensor(full, device="cuda")
    S = overlap(wctx, t[:, :2500])   # row stride 3000, length 2500
    ref = oracle.overlap(np.ascontiguousarray(full[:, :2500]))
    assert np.abs(S.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-13


@pytest.mark.parametrize("method", ["cholesky", "loewdin"])
def test_orthonormalize(oracle, torch_cuda, wctx, method):
    torch = torch_cuda
    rng = np.random.default_rng(3)
    psi = torch.tensor(rng.uniform(-1, 1, (32, 20000)), device="cuda")
    psi, S = orthonormalize(wctx, psi, method)
    S2 = overlap(wctx, psi)
    assert (S2 - torch.eye(32, device="cuda", dtype=torch.float64)).abs().max().item() < 1e-12
    if method == "cholesky":
        Lref = oracle.cholesky_lower(S.cpu().numpy())
        Lgpu = torch.linalg.cholesky(S).cpu().numpy()
        assert np.abs(Lgpu - Lref).max() / np.abs(Lref).max() < 1e-12


@pytest.mark.parametrize("dtype_name,ld", [("float64", 3001), ("float32", 5001)])
def test_overlap_unaligned_rows(oracle, torch_cuda, wctx, dtype_name, ld):
    """Row strides that are not 16-byte multiples take the element-copy path."""
    torch = torch_cuda
    rng = np.random.default_rng(ld)
    full = rng.uniform(-1, 1, (70, ld))
    dt = getattr(torch, dtype_name)
    t = torch.tensor(full, dtype=dt, device="cuda")
    K = ld - 37
    S = overlap(wctx, t[:, :K]).cpu().numpy()
    src = full[:, :K].astype(np.float32).astype(np.float64) if dtype_name == "float32" else full[:, :K]
    ref = oracle.overlap(np.ascontiguousarray(src))
    assert np.abs(S - ref).max() / np.abs(ref).max() < 1e-13


@pytest.mark.parametrize("norb,K,dtype_name", [(7, 1000, "float64"), (100, 12345, "float64"), (130, 9001, "float32")])
def test_subspace_matrix_matches_gemm(torch_cuda, wctx, norb, K, dtype_name):
    """L = <psi_i|hpsi_j> on every tile of the square (subspace_matrix,
    orthogonality.f90:196-224), non-symmetric, FP32 rows widened."""
    from wvlh.ortho import subspace_matrix
    torch = torch_cuda
    rng = np.random.default_rng(norb)
    a, b = rng.uniform(-1, 1, (norb, K)), rng.uniform(-1, 1, (norb, K))
    if dtype_name == "float32":
        a, b = a.astype(np.float32).astype(np.float64), b.astype(np.float32).astype(np.float64)
    dt = getattr(torch, dtype_name)
    L = subspace_matrix(wctx, torch.tensor(a, dtype=dt, device="cuda"), torch.tensor(b, dtype=dt, device="cuda"))
    ref = a @ b.T
    assert np.abs(L.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-13


@pytest.mark.parametrize("occ", ["equal", "mixed"])
def test_orthoconstraint_matches_oracle(oracle, torch_cuda, wctx, occ):
    from wvlh.ortho import orthoconstraint
    torch = torch_cuda
    rng = np.random.default_rng(5)
    norb, K = 40, 20000
    psi = rng.uniform(-1, 1, (norb, K))
    hpsi = rng.uniform(-1, 1, (norb, K))
    f = np.full(norb, 2.0) if occ == "equal" else rng.choice([2.0, 1.0, 0.0], norb)
    g_ref, lam, tr, asy, mix = oracle.orthoconstraint(psi, hpsi, f)
    tp, th = torch.tensor(psi, device="cuda"), torch.tensor(hpsi, device="cuda")
    L, tr2, asy2, mix2 = orthoconstraint(wctx, tp, th, occup=f)
    assert np.abs(L.cpu().numpy() - lam).max() / np.abs(lam).max() < 1e-13
    assert np.abs(th.cpu().numpy() - g_ref).max() / np.abs(g_ref).max() < 1e-13
    assert abs(tr2 - tr) <= 1e-12 * abs(tr) and abs(asy2 - asy) <= 1e-12 * asy and abs(mix2 - mix) <= 1e-12 * max(mix, 1e-300)


def test_overlap_sharded_single_process_uses_the_device_kernel(torch_cuda, wctx):
    """Without a process group the sharded overlap is the library's overlap of
    the local rows (the multi-rank exchange is covered by the gloo tests)."""
    from wvlh.shard import overlap_sharded
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(3)
    X = torch.rand(40, 3001, generator=g, dtype=torch.float64, device="cuda") * 2 - 1
    S = overlap_sharded(X, ctx=wctx)
    ref = (X.cpu().numpy() @ X.cpu().numpy().T)
    assert np.abs(S.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("norb,K,lower,beta", [(64, 4096, False, 0.0), (37, 5003, True, 0.0), (100, 12345, False, 1.0),
                                               (256, 30000, True, 0.0), (33, 777, False, 1.0)])
def test_panel_apply_matches_fp64_product(torch_cuda, wctx, norb, K, lower, beta):
    """out = beta out + alpha M psi on the tensor-core panel apply against the
    FP64 product on the host (odd orbital counts and lengths take the
    one-double copies; lower skips the slices above the diagonal)."""
    from wvlh.ortho import panel_apply
    torch = torch_cuda
    rng = np.random.default_rng(norb * K)
    M = rng.uniform(-1, 1, (norb, norb))
    if lower:
        M = np.tril(M)
    psi = rng.uniform(-1, 1, (norb, K))
    out0 = rng.uniform(-1, 1, (norb, K))
    alpha = -0.75
    tout = torch.tensor(out0, device="cuda")
    panel_apply(wctx, torch.tensor(M, device="cuda"), torch.tensor(psi, device="cuda"), out=tout, alpha=alpha,
                beta=beta, lower=lower)
    ref = beta * out0 + alpha * (M @ psi)
    assert np.abs(tout.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-13


@pytest.mark.parametrize("method", ["cholesky", "loewdin"])
def test_orthonormalize_matches_oracle_chain(oracle, torch_cuda, wctx, method):
    """psi <- L^-1 psi (dpotrf, dtrtri, dtrmm) or S^-1/2 psi on the panel
    apply against the same steps in FP64 on the host from the oracle's S."""
    torch = torch_cuda
    rng = np.random.default_rng(11)
    norb, K = 48, 30011
    psi = rng.uniform(-1, 1, (norb, K))
    t = torch.tensor(psi, device="cuda")
    orthonormalize(wctx, t, method)
    S = oracle.overlap(psi)
    if method == "cholesky":
        M = np.linalg.inv(oracle.cholesky_lower(S))
    else:
        w, U = np.linalg.eigh(S)
        M = (U / np.sqrt(w)) @ U.T
    ref = M @ psi
    assert np.abs(t.cpu().numpy() - ref).max() / np.abs(ref).max() < 1e-11
