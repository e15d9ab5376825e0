"""CPU tests of the free-boundary bounds (make_bounds / make_all_ib,
locregs/bounds.f90:690-1135) restated in wvlh.keys.

The reference's bounded grow passes (growshrink.f90:12-48) write the
real-space array only inside the spans make_all_ib derives and leave
"nonphysical values" elsewhere; apply_potential_lr_bounds then visits the
real-space span ibyyzz_r only.  This library's free-BC passes are dense.
They agree with the bounded ones exactly when the dense result is zero
outside the spans, which these tests check on the oracle's dense
synthesis + magic filter for irregular coarse and fine regions."""
import numpy as np
import pytest

from wvlh.keys import Locreg, make_all_ib, make_bounds


def test_make_bounds_first_last_and_sentinels():
    rng = np.random.default_rng(0)
    m = rng.random((5, 6, 7)) < 0.3
    m[2, 3, :] = False
    ibyz, ibxz, ibxy = make_bounds(m)
    for i3 in range(5):
        for i2 in range(6):
            idx = np.nonzero(m[i3, i2, :])[0]
            want = (idx[0], idx[-1]) if len(idx) else (1000, -1000)
            assert ibyz.get(i2, i3) == want
    for i3 in range(5):
        for i1 in range(7):
            idx = np.nonzero(m[i3, :, i1])[0]
            assert ibxz.get(i1, i3) == ((idx[0], idx[-1]) if len(idx) else (1000, -1000))
    for i2 in range(6):
        for i1 in range(7):
            idx = np.nonzero(m[:, i2, i1])[0]
            assert ibxy.get(i1, i2) == ((idx[0], idx[-1]) if len(idx) else (1000, -1000))


def ellipsoid(N, frac, shift=(0.0, 0.0, 0.0)):
    idx = np.meshgrid(*[np.arange(v) for v in N[::-1]], indexing="ij")
    r2 = np.zeros(N[::-1])
    for ax, n, s in zip(idx, N[::-1], shift[::-1]):
        r2 += ((ax - (n - 1) / 2.0 - s) / (frac * n)) ** 2
    return r2 <= 1.0


CASES = [((12, 10, 14), 0.55, 0.3, (0.0, 0.0, 0.0)), ((9, 13, 11), 0.6, 0.25, (1.0, -1.5, 0.5)),
         ((16, 8, 10), 0.5, 0.35, (-2.0, 0.5, 1.0))]


@pytest.mark.parametrize("N,fc,ff,shift", CASES)
def test_dense_grow_vanishes_outside_bounds(oracle, N, fc, ff, shift):
    mc = ellipsoid(N, fc, shift)
    mf = ellipsoid(N, ff, shift) & mc
    lr = Locreg.from_masks(mc, mf, (0, 0, 0), (0.45, 0.45, 0.45))
    n = tuple(v - 1 for v in N)
    fz, fy, fx = np.nonzero(mf)
    nfl, nfu = (fx.min(), fy.min(), fz.min()), (fx.max(), fy.max(), fz.max())
    ibyz_c, ibxz_c, ibxy_c = make_bounds(mc)
    ibyz_f, ibxz_f, ibxy_f = make_bounds(mf)
    ib = make_all_ib(n, nfl, nfu, ibxy_c, ibxy_f, ibyz_c, ibyz_f)
    d = oracle.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
    rng = np.random.default_rng(sum(N))
    pc, pf = rng.uniform(-1, 1, lr.nvctr_c), rng.uniform(-1, 1, 7 * lr.nvctr_f)
    I1, I2, I3 = lr.isf
    for part, ibx in (("coarse", ib["ibxxyy_c"]), ("fine", ib["ibxxyy_f"])):
        c = pc if part == "coarse" else np.zeros_like(pc)
        f = pf if part == "fine" else np.zeros_like(pf)
        psir = oracle.magic(d, oracle.synthese(d, oracle.uncompress(d, c, f))).reshape(I3, I2, I1)
        # the last grow pass writes, per (I1, I2) column, I3 = 2 lo - 14 .. 2 hi + 16
        written = np.zeros((I3, I2, I1), bool)
        for a in range(ibx.lo.shape[1]):
            for b in range(ibx.lo.shape[0]):
                lo, hi = ibx.lo[b, a], ibx.hi[b, a]
                if lo > hi:
                    continue
                Ia, Ib = a + ibx.a0, b + ibx.b0     # (I1, I2), -14-based
                written[2 * lo - 14 + 14:2 * hi + 16 + 15, Ib + 14, Ia + 14] = True
        assert np.abs(psir).max() > 0
        assert np.all(psir[~written] == 0.0), part
    # real space: per (I2, I3) line the potential step visits ibyyzz_r (0-based ISF index)
    psir = oracle.magic(d, oracle.synthese(d, oracle.uncompress(d, pc, pf))).reshape(I3, I2, I1)
    r = ib["ibyyzz_r"]
    inside = np.zeros_like(psir, bool)
    for a in range(r.lo.shape[1]):
        for b in range(r.lo.shape[0]):
            if r.lo[b, a] <= r.hi[b, a]:
                inside[b, a, r.lo[b, a]:r.hi[b, a] + 1] = True
    assert np.all(psir[~inside] == 0.0)
    # the spans are tight enough to matter: a real part of the box is skipped
    assert (~inside).mean() > 0.02


@pytest.mark.parametrize("periodic,center,locrad", [((0, 0, 0), (3.1, 2.7, 3.4), 2.3),
                                                     ((1, 1, 1), (0.4, 5.2, 0.3), 2.0),
                                                     ((1, 0, 1), (5.5, 2.0, 0.1), 1.7)])
def test_segkeys_sphere_against_direct_mask(periodic, center, locrad):
    """segkeys_Sphere of a full global box: the local segments cover exactly
    the cells within locrad (periodic images included), each local segment a
    run along x of the local box, offsets consistent with the segment sizes."""
    from wvlh.keys import segkeys, segkeys_sphere
    N = (14, 12, 13)
    h = (0.45, 0.5, 0.42)
    kg, kv = segkeys(np.ones(N[::-1], bool))
    n = tuple(v - 1 for v in N)
    # the local box: every image cell within locrad, brute force
    cells = []
    for i3 in range(N[2]):
        for i2 in range(N[1]):
            for i1 in range(N[0]):
                for a3 in ((-1, 0, 1) if periodic[2] else (0,)):
                    for a2 in ((-1, 0, 1) if periodic[1] else (0,)):
                        for a1 in ((-1, 0, 1) if periodic[0] else (0,)):
                            j = (i1 + a1 * N[0], i2 + a2 * N[1], i3 + a3 * N[2])
                            if sum((j[d] * h[d] - center[d]) ** 2 for d in range(3)) <= locrad ** 2:
                                cells.append(j)
    cells = np.array(cells)
    nl, nu = cells.min(axis=0), cells.max(axis=0)
    kgl, kvl, kgg, kvg, nvctr = segkeys_sphere(n, periodic, (0, 0, 0), tuple(nl), tuple(nu), h, locrad, center, kg)
    assert nvctr == len(cells)
    # local keys: sorted, each within one local x-line, covering exactly the cells
    Ll = nu - nl + 1
    got = set()
    for (a, b) in kgl:
        assert (a - 1) // Ll[0] == (b - 1) // Ll[0]
        for g in range(a - 1, b):
            i3, r = divmod(g, Ll[0] * Ll[1])
            i2, i1 = divmod(r, Ll[0])
            got.add((i1 + nl[0], i2 + nl[1], i3 + nl[2]))
    assert got == set(map(tuple, cells))
    assert np.all(np.diff(kgl[:, 0]) > 0)
    # offsets: in visiting order they are cumulative; the sorted copy permutes them
    sizes = kgg[:, 1] - kgg[:, 0] + 1
    assert np.array_equal(kvg, 1 + np.concatenate([[0], np.cumsum(sizes)[:-1]]))
    assert sorted(kvl.tolist()) == sorted(kvg.tolist())
    if not any(periodic):
        assert np.array_equal(kvl, kvg)
