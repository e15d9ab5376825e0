"""CPU checks of the compressed scalar product (the reference's wpdot,
wavelib/scalprod.f90:3222) as the oracle restates it.

* Where every b segment meets at most one a segment (convex regions, the
  projector-inside-wavefunction case the reference uses it for), wpdot is
  the plain sum over the grid points both vectors carry.
* In general it is the per-segment rule the GPU kernel implements: each b
  segment takes its overlap with the first a segment it meets, and b segments
  after the first one that starts past a's last segment start are skipped.
"""
import numpy as np
import pytest

from wvlh.keys import segkeys


def rule(ka, a, kb, b):
    """Independent restatement of the per-b-segment rule, in numpy."""
    def part(kga, kva, pa, kgb, kvb, pb, nc):
        s = np.zeros(nc)
        if len(kva) == 0:
            return s
        sa, ea = kga[:, 0], kga[:, 1]
        last = sa[-1]
        for ib in range(len(kvb)):
            kbs, kbe = kgb[ib]
            if ib > 0 and kgb[ib - 1, 0] > last:
                continue   # the reference's search index is past the end
            jb0 = max(kbs, sa[0])
            i = int(np.searchsorted(sa, jb0, side="right")) - 1
            if ea[i] < jb0:
                i += 1
                if i >= len(sa) or sa[i] > kbe:
                    continue
                jb0 = sa[i]
            n = min(kbe, ea[i]) - jb0 + 1
            if n <= 0:
                continue
            a0 = kva[i] - 1 + (jb0 - sa[i])
            b0 = kvb[ib] - 1 + (jb0 - kbs)
            s += (pa[a0:a0 + n] * pb[b0:b0 + n]).sum(axis=0)
        return s

    nca = int((ka[0][:, 1] - ka[0][:, 0] + 1).sum())
    ncb = int((kb[0][:, 1] - kb[0][:, 0] + 1).sum())
    sc = part(ka[0], ka[1], a[:nca, None], kb[0], kb[1], b[:ncb, None], 1)
    sf = part(ka[2], ka[3], a[nca:].reshape(-1, 7), kb[2], kb[3], b[ncb:].reshape(-1, 7), 7)
    return sc.sum() + sf.sum()


def dense(k, v, N):
    """Coefficients on the box: (N3, N2, N1) coarse and (N3, N2, N1, 7) fine."""
    c = np.zeros(N[::-1])
    f = np.zeros(N[::-1] + (7,))
    nc = 0
    for (j0, j1), kv in zip(k[0], k[1]):
        c.reshape(-1)[j0 - 1:j1] = v[kv - 1:kv - 1 + j1 - j0 + 1]
        nc += j1 - j0 + 1
    vf = v[nc:].reshape(-1, 7)
    for (j0, j1), kv in zip(k[2], k[3]):
        f.reshape(-1, 7)[j0 - 1:j1] = vf[kv - 1:kv - 1 + j1 - j0 + 1]
    return c, f


def masks(rng, N, pc, pf):
    m = rng.random(N[::-1]) < pc
    return m, m & (rng.random(N[::-1]) < pf)


@pytest.mark.parametrize("seed", range(12))
def test_oracle_equals_per_segment_rule(oracle, seed):
    rng = np.random.default_rng(seed)
    N = tuple(int(v) for v in rng.integers(5, 12, 3))
    ma, fa = masks(rng, N, rng.uniform(0.3, 0.9), 0.5)
    mb, fb = masks(rng, N, rng.uniform(0.3, 0.9), 0.5)
    ka, kb = segkeys(ma) + segkeys(fa), segkeys(mb) + segkeys(fb)
    a = rng.uniform(-1, 1, int(ma.sum() + 7 * fa.sum()))
    b = rng.uniform(-1, 1, int(mb.sum() + 7 * fb.sum()))
    got = oracle.wpdot(ka, a, kb, b)
    assert abs(got - rule(ka, a, kb, b)) <= 1e-13 * max(1.0, abs(got))


def test_convex_regions_give_the_grid_sum(oracle):
    """Boxes (one run per x-line each): wpdot = sum over the common points."""
    N = (14, 12, 10)
    rng = np.random.default_rng(3)
    ma = np.zeros(N[::-1], bool)
    ma[1:9, 2:11, 3:13] = True
    mb = np.zeros(N[::-1], bool)
    mb[4:10, 0:8, 0:9] = True
    fa, fb = ma.copy(), mb.copy()
    fa[:, :, 10:] = False
    fb[:, :, :2] = False
    ka, kb = segkeys(ma) + segkeys(fa), segkeys(mb) + segkeys(fb)
    a = rng.uniform(-1, 1, int(ma.sum() + 7 * fa.sum()))
    b = rng.uniform(-1, 1, int(mb.sum() + 7 * fb.sum()))
    ca, fa_ = dense(ka, a, N)
    cb, fb_ = dense(kb, b, N)
    ref = (ca * cb).sum() + (fa_ * fb_).sum()
    assert abs(oracle.wpdot(ka, a, kb, b) - ref) <= 1e-13 * abs(ref)


def test_only_the_first_overlapping_a_segment_counts(oracle):
    """A b run over a gap of a: the reference counts the first a run only."""
    N = (12, 1, 1)
    ma = np.zeros((1, 1, 12), bool)
    ma[0, 0, [1, 2, 3, 6, 7]] = True      # a runs [2..4] and [7..8] (1-based)
    mb = np.zeros((1, 1, 12), bool)
    mb[0, 0, 0:10] = True                 # one b run [1..10]
    none = np.zeros((1, 1, 12), bool)
    ka, kb = segkeys(ma) + segkeys(none), segkeys(mb) + segkeys(none)
    a = np.arange(1.0, 6.0)               # values at points 2, 3, 4, 7, 8
    b = np.ones(10)
    assert oracle.wpdot(ka, a, kb, b) == 1.0 + 2.0 + 3.0
