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
