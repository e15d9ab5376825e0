"""Segment keys of a compressed wavelet descriptor.

The reference stores a wavefunction on a localisation region as runs
("segments") of occupied coarse cells along x: ``keyg(2,nseg)`` holds the
1-based first/last linear index of each run in the ``(n1+1)(n2+1)(n3+1)`` box
(x fastest) and ``keyv(nseg)`` its 1-based offset in the compressed vector
(``bigdft/src/locregs/compression.f90:29-39``).  :func:`segkeys` computes them
from a logical mask exactly like ``num_segkeys``/``segkeys``
(``bigdft/src/locregs/initlocregs.f90:1573-1687``): a run ends at the last
occupied cell of a line, so segments never cross lines.
"""
from dataclasses import dataclass, field

import numpy as np


def segkeys(mask):
    """mask[i3, i2, i1] -> (keyg int32 (nseg, 2), keyv int32 (nseg,)), 1-based."""
    m = np.ascontiguousarray(mask, dtype=bool)
    n3, n2, n1 = m.shape
    lines = m.reshape(n3 * n2, n1).astype(np.int8)
    pad = np.zeros((lines.shape[0], 1), np.int8)
    d = np.diff(np.concatenate([pad, lines, pad], axis=1), axis=1)
    ls, i_start = np.nonzero(d == 1)           # run starts (row-major: sorted by line then i1)
    le, i_end = np.nonzero(d == -1)            # one past run ends
    assert np.array_equal(ls, le)
    base = ls.astype(np.int64) * n1            # line index = i3*n2 + i2
    keyg = np.empty((len(ls), 2), np.int32)
    keyg[:, 0] = base + i_start + 1
    keyg[:, 1] = base + i_end                  # (i_end - 1) + 1
    lens = i_end - i_start
    keyv = np.empty(len(ls), np.int32)
    if len(ls):
        keyv[0] = 1
        keyv[1:] = 1 + np.cumsum(lens[:-1])
    return keyg, keyv


@dataclass
class Locreg:
    """A localisation region: coarse cells per dimension (n1+1, n2+1, n3+1),
    periodicity, coarse grid spacing, coarse and fine keys."""
    n: tuple
    periodic: tuple
    hgrid: tuple
    keyg_c: np.ndarray
    keyv_c: np.ndarray
    keyg_f: np.ndarray
    keyv_f: np.ndarray
    nvctr_c: int = field(init=False)
    nvctr_f: int = field(init=False)

    def __post_init__(self):
        self.keyg_c = np.ascontiguousarray(self.keyg_c, np.int32).reshape(-1, 2)
        self.keyg_f = np.ascontiguousarray(self.keyg_f, np.int32).reshape(-1, 2)
        self.keyv_c = np.ascontiguousarray(self.keyv_c, np.int32)
        self.keyv_f = np.ascontiguousarray(self.keyv_f, np.int32)
        self.nvctr_c = int((self.keyg_c[:, 1] - self.keyg_c[:, 0] + 1).sum())
        self.nvctr_f = int((self.keyg_f[:, 1] - self.keyg_f[:, 0] + 1).sum())

    @classmethod
    def from_masks(cls, mask_c, mask_f, periodic, hgrid):
        kc, vc = segkeys(mask_c)
        kf, vf = segkeys(mask_f)
        return cls(tuple(int(v) for v in mask_c.shape[::-1]), tuple(int(p) for p in periodic),
                   tuple(float(h) for h in hgrid), kc, vc, kf, vf)

    @property
    def ncoeff(self):
        return self.nvctr_c + 7 * self.nvctr_f

    @property
    def fine(self):
        return tuple(2 * n if p else 2 * n + 14 for n, p in zip(self.n, self.periodic))

    @property
    def isf(self):
        """ISF (real-space) grid extents, x first: 2N periodic, 2N+29 free."""
        return tuple(2 * n if p else 2 * n + 29 for n, p in zip(self.n, self.periodic))

    @property
    def nisf(self):
        a, b, c = self.isf
        return a * b * c

    @property
    def coarse_cells(self):
        a, b, c = self.n
        return a * b * c


# ---------------------------------------------------------------------------
# Bounds of the free-boundary grow / shrink passes (locregs/bounds.f90)
#
# The reference's free-BC convolutions visit, along each line, only the span
# between the first and last occupied point, and record those spans once per
# region: make_bounds gives them for the coarse and fine masks, make_all_ib
# derives the spans of every intermediate array of the grow (synthesis +
# magic filter, growshrink.f90:12-48) and shrink passes and of the real-space
# array.  Points outside the spans are never written by the bounded passes
# ("nonphysical values", growshrink.f90:42-48); the dense passes of this
# library compute them, and they are exactly zero there (the support of the
# grown function lies inside the spans), which the tests check.
#
# Arrays follow the Fortran layout ib(2, a, b) as numpy arrays of shape
# (nb, na, 2) (b slowest), each index range starting at the offset returned
# beside it: a Bounds2 holds lo = ib[..., 0], hi = ib[..., 1] and the first
# index of each axis.  Empty lines hold the reference's sentinels 1000/-1000.


@dataclass
class Bounds2:
    """ib(2, a0:a1, b0:b1): lo/hi of shape (nb, na), first indices (a0, b0)."""
    lo: np.ndarray
    hi: np.ndarray
    a0: int
    b0: int

    def get(self, a, b):
        return int(self.lo[b - self.b0, a - self.a0]), int(self.hi[b - self.b0, a - self.a0])


def _first_last(logrid, axis, start):
    """First / last index (offset by start) along axis where logrid is set,
    1000 / -1000 where no point is (bounds.f90:707-724, ib_from_logrid)."""
    n = logrid.shape[axis]
    any_ = logrid.any(axis=axis)
    first = np.argmax(logrid, axis=axis) + start
    last = n - 1 - np.argmax(np.flip(logrid, axis=axis), axis=axis) + start
    return np.where(any_, first, 1000).astype(np.int64), np.where(any_, last, -1000).astype(np.int64)


def make_bounds(logrid):
    """make_bounds (locregs/bounds.f90:690-774) of logrid[i3, i2, i1]:
    ibyz(2, 0:n2, 0:n3) (span along i1), ibxz(2, 0:n1, 0:n3) (along i2),
    ibxy(2, 0:n1, 0:n2) (along i3)."""
    g = np.asarray(logrid, bool)
    lo, hi = _first_last(g, 2, 0)                    # (i3, i2)
    ibyz = Bounds2(lo, hi, 0, 0)
    lo, hi = _first_last(g, 1, 0)                    # (i3, i1)
    ibxz = Bounds2(lo, hi, 0, 0)
    lo, hi = _first_last(g, 0, 0)                    # (i2, i1)
    ibxy = Bounds2(lo, hi, 0, 0)
    return ibyz, ibxz, ibxy


def _grow_mark(ib, lo_out, n_out):
    """ib_to_logrid(_rot/_inv) (bounds.f90:887-907,1012-1032): for every line
    of ib, mark the points 2 lo - 14 .. 2 hi + 16 of a new axis whose first
    index is lo_out (n_out points); returns a boolean array (lines..., n_out)."""
    idx = np.arange(n_out)[None, :] + lo_out
    lo = ib.lo.reshape(-1, 1)
    hi = ib.hi.reshape(-1, 1)
    m = (idx >= 2 * lo - 14) & (idx <= 2 * hi + 16)
    return m.reshape(ib.lo.shape + (n_out,))


def _squares(b):
    """squares (bounds.f90:1102-1135): merge the spans of each 2 x 2 block of
    lines (pairs of a starting at the array's first index, likewise b); a
    dimension of extent 1 (n = 0 in the reference) leaves the array alone."""
    nb, na = b.lo.shape
    if na == 1 or nb == 1:
        return
    for jb in range(0, nb - 1, 2):
        for ja in range(0, na - 1, 2):
            blo = b.lo[jb:jb + 2, ja:ja + 2]
            bhi = b.hi[jb:jb + 2, ja:ja + 2]
            blo[...] = blo.min()
            bhi[...] = bhi.max()


def _squares_1d(b):
    """squares_1d (bounds.f90:1076-1099): merge the spans of pairs of lines
    along the first axis a only."""
    nb, na = b.lo.shape
    for ja in range(0, na - 1, 2):
        sl = slice(ja, ja + 2)
        b.lo[:, sl] = b.lo[:, sl].min(axis=1, keepdims=True)
        b.hi[:, sl] = b.hi[:, sl].max(axis=1, keepdims=True)


def make_all_ib(n, nfl, nfu, ibxy_c, ibxy_f, ibyz_c, ibyz_f):
    """make_all_ib (locregs/bounds.f90:777-862) for a box of n = (n1, n2, n3)
    (the reference's n = cells - 1) and fine region nfl..nfu.  Inputs are the
    make_bounds spans of the coarse and fine masks (ibyz_c is squared in
    place, as make_ib_c does).  Returns a dict of Bounds2:
    shrink: ibzzx_c(2, -14:2n3+16, 0:n1), ibyyzz_c(2, -14:2n2+16, -14:2n3+16),
            ibxy_ff, ibzzx_f, ibyyzz_f (fine-region ranges);
    grow:   ibzxx_c(2, 0:n3, -14:2n1+16), ibxxyy_c(2, -14:2n1+16, -14:2n2+16),
            ibyz_ff, ibzxx_f, ibxxyy_f;
    real space: ibyyzz_r(2, -14:2n2+16, -14:2n3+16)."""
    n1, n2, n3 = n
    nfl1, nfl2, nfl3 = nfl
    nfu1, nfu2, nfu3 = nfu
    out = {}

    def fine_sub(b, a0, a1, b0, b1):
        return Bounds2(b.lo[b0 - b.b0:b1 - b.b0 + 1, a0 - b.a0:a1 - b.a0 + 1].copy(),
                       b.hi[b0 - b.b0:b1 - b.b0 + 1, a0 - b.a0:a1 - b.a0 + 1].copy(), a0, b0)

    def ib_inv(ibxy, l1, u1, l2, u2, l3, u3):
        # make_ib_inv (bounds.f90:865-884): spans along i3 -> marks on I3,
        # spans along i2 per (I3, i1) -> marks on I2, spans along i1 per (I2, I3)
        m1 = _grow_mark(ibxy, 2 * l3 - 14, 2 * (u3 - l3) + 31)       # (i2, i1, I3)
        lo, hi = _first_last(m1, 0, l2)                                # (i1, I3) -> ibzzx(2, I3, i1)
        ibzzx = Bounds2(lo, hi, 2 * l3 - 14, l1)
        m2 = _grow_mark(ibzzx, 2 * l2 - 14, 2 * (u2 - l2) + 31)       # (i1, I3, I2)
        lo, hi = _first_last(m2, 0, l1)                                # (I3, I2) -> ibyyzz(2, I2, I3)
        return ibzzx, Bounds2(lo, hi, 2 * l2 - 14, 2 * l3 - 14)

    def ib_grow(ibyz, l1, u1, l2, u2, l3, u3, square):
        # make_ib_c / make_ib (bounds.f90:937-1009): spans along i1 -> marks on
        # I1, spans along i2 per (i3, I1) -> marks on I2, spans along i3 per (I1, I2)
        if square:
            _squares(ibyz)
        m1 = _grow_mark(ibyz, 2 * l1 - 14, 2 * (u1 - l1) + 31)       # (i3, i2, I1)
        lo, hi = _first_last(m1, 1, l2)                                # (i3, I1) -> ibzxx(2, i3, I1)
        ibzxx = Bounds2(lo.T.copy(), hi.T.copy(), l3, 2 * l1 - 14)     # stored (I1, i3)
        if square:
            _squares(ibzxx)
        m2 = _grow_mark(ibzxx, 2 * l2 - 14, 2 * (u2 - l2) + 31)       # (I1, i3, I2)
        lo, hi = _first_last(m2, 1, l3)                                # (I1, I2) -> ibxxyy(2, I1, I2)
        ibxxyy = Bounds2(lo.T.copy(), hi.T.copy(), 2 * l1 - 14, 2 * l2 - 14)   # stored (I2, I1)
        if square:
            _squares(ibxxyy)
        return ibzxx, ibxxyy

    # shrink
    ibxy_ff = fine_sub(ibxy_f, nfl1, nfu1, nfl2, nfu2)
    out["ibxy_ff"] = ibxy_ff
    out["ibzzx_c"], out["ibyyzz_c"] = ib_inv(ibxy_c, 0, n1, 0, n2, 0, n3)
    out["ibzzx_f"], out["ibyyzz_f"] = ib_inv(ibxy_ff, nfl1, nfu1, nfl2, nfu2, nfl3, nfu3)
    # real space (bounds.f90:831-844): twice the coarse shrink span, widened by 30
    c = out["ibyyzz_c"]
    keep = c.lo != 1000
    r = Bounds2(np.where(keep, 2 * c.lo, 1000), np.where(keep, 2 * c.hi + 30, -1000), -14, -14)
    _squares(r)
    out["ibyyzz_r"] = r
    # grow
    ibyz_ff = fine_sub(ibyz_f, nfl2, nfu2, nfl3, nfu3)
    out["ibyz_ff"] = ibyz_ff
    out["ibzxx_c"], out["ibxxyy_c"] = ib_grow(ibyz_c, 0, n1, 0, n2, 0, n3, True)
    out["ibzxx_f"], out["ibxxyy_f"] = ib_grow(ibyz_ff, nfl1, nfu1, nfl2, nfu2, nfl3, nfu3, False)
    _squares_1d(out["ibxxyy_f"])
    return out


def segkeys_sphere(n, periodic, nl_glob, nl, nu, hgrid, locrad, center, keyg_glob_in):
    """Keys of a localisation region cut from a global region by a sphere:
    num_segkeys_sphere + segkeys_Sphere (locregs/initlocregs.f90:140-727).

    n = (n1, n2, n3): the global box is (n1+1)(n2+1)(n3+1) coarse cells, its
    segments keyg_glob_in (nseg, 2), 1-based, x fastest, the box starting at
    nl_glob.  A global point is inside when one of its periodic images (one
    box length either way along periodic axes) lies within locrad of center
    (positions i*h, as the reference takes them); that image's cell, relative
    to the local box nl..nu, is its local cell.  Runs of consecutive inside
    points of one global segment make the local segments.

    Returns (keyg_loc, keyv_loc, keyg_glob, keyv_glob, nvctr): keyg_glob/keyv_glob
    in the order the global segments are visited (the compressed vector's
    order); keyg_loc sorted by local start index with keyv_loc giving each
    segment's 1-based offset in that same vector (the reference's minloc sort)."""
    n1, n2, n3 = n
    nl1g, nl2g, nl3g = nl_glob
    nl1, nl2, nl3 = nl
    nu1, nu2, nu3 = nu
    hx, hy, hz = hgrid
    cut = locrad ** 2
    n1p1, np_ = n1 + 1, (n1 + 1) * (n2 + 1)
    n1lp1 = nu1 - nl1 + 1
    nlp = n1lp1 * (nu2 - nl2 + 1)
    imgs = [(-1, 0, 1) if p else (0,) for p in periodic]
    loc_starts, loc_ends, glob_starts, glob_ends, vstart = [], [], [], [], []
    nvctr = 0
    for j0, j1 in np.asarray(keyg_glob_in).reshape(-1, 2):
        ii = int(j0) - 1
        i3 = ii // np_
        ii -= i3 * np_
        i2 = ii // n1p1
        i0 = ii - i2 * n1p1
        i1 = i0 + int(j1) - int(j0)
        ii2, ii3 = i2 + nl2g, i3 + nl3g
        base = ii3 * np_ + ii2 * n1p1 + 1
        seg = False
        igp = None
        for i in range(i0, i1 + 1):
            ii1 = i + nl1g
            inside, hit = False, None
            for a3 in imgs[2]:
                jj3 = ii3 + a3 * (n3 + 1)
                dz = (jj3 * hz - center[2]) ** 2
                for a2 in imgs[1]:
                    jj2 = ii2 + a2 * (n2 + 1)
                    dy = (jj2 * hy - center[1]) ** 2
                    for a1 in imgs[0]:
                        jj1 = ii1 + a1 * (n1 + 1)
                        dx = (jj1 * hx - center[0]) ** 2
                        if dx + dy + dz <= cut:
                            if inside:
                                raise ValueError("two periodic images inside the sphere (locrad too large)")
                            inside, hit = True, (jj1, jj2, jj3)
            if inside:
                jj1, jj2, jj3 = hit
                if not (nl1 <= jj1 <= nu1 and nl2 <= jj2 <= nu2 and nl3 <= jj3 <= nu3):
                    raise ValueError("inside point outside the local box")
                igp = (jj3 - nl3) * nlp + (jj2 - nl2) * n1lp1 + (jj1 - nl1) + 1
                nvctr += 1
                if not seg:
                    loc_starts.append(igp)
                    glob_starts.append(base + ii1)
                    vstart.append(nvctr)
                    seg = True
            elif seg:
                loc_ends.append(igp)
                glob_ends.append(base + ii1 - 1)
                seg = False
        if seg:
            loc_ends.append(igp)
            glob_ends.append(base + i1 + nl1g)
    keyg_glob = np.array([glob_starts, glob_ends], np.int64).T.reshape(-1, 2).astype(np.int32)
    keyv_glob = np.array(vstart, np.int32)
    keyg_l = np.array([loc_starts, loc_ends], np.int64).T.reshape(-1, 2)
    order = np.argsort(keyg_l[:, 0], kind="stable")
    return keyg_l[order].astype(np.int32), keyv_glob[order], keyg_glob, keyv_glob, nvctr
