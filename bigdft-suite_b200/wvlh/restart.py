"""Wavefunction files in the reference's restart formats.

One orbital per file, as writeonewave (bigdft/src/modules/io.f90:2639-2724)
writes it and io_read_descr / read_psi_compress (:1616-1790) read it back:

    iorb, eval
    hx, hy, hz
    n1, n2, n3                      (maximum coarse indices)
    nat
    x, y, z                         (one line per atom)
    nvctr_c, nvctr_f
    i1 i2 i3 c                      (coarse points, in key order)
    i1 i2 i3 f1 .. f7               (fine points, in key order)

"Plain" files are formatted: the header lines list-directed, the atoms
'(3(1x,e24.17))', the coarse points '(3(i4),1x,e19.12)', the fine points
'(3(i4),7(1x,e17.10))'.  "Binary" files are Fortran sequential unformatted,
one record per line above (4-byte length markers around each record; int32
integers, float64 reals).  File names follow filename_of_iorb
(restart.f90:512-596): <radical>-k001-NR.b000001, or .bin.b000001.

The server uses these files to move a client's orbitals out of device memory
and back (Server.evict / Server.restore).
"""
import re
import struct

import numpy as np

from ._lib import WvlhError


def fortran_e(x, w, d):
    """Fortran Ew.d: a sign or blank, 0., d digits, E and a signed two-digit
    exponent (three digits replace the E when the exponent needs them)."""
    x = float(x)
    if x == 0.0 or not np.isfinite(x):
        body = "0." + "0" * d + "E+00" if x == 0.0 else repr(x)
        s = ("-" if np.signbit(x) and x == 0.0 else "") + body
        return s.rjust(w)
    m, e = ("%.*e" % (d - 1, abs(x))).split("e")
    digits = m.replace(".", "")
    ex = int(e) + 1
    tail = ("E%+03d" % ex) if abs(ex) < 100 else ("%+04d" % ex)
    s = ("-" if x < 0 else "") + "0." + digits + tail
    if len(s) > w:
        return "*" * w
    return s.rjust(w)


def wave_filename(radical, iorb, binary=False, ikpt=1, spin="N", part="R"):
    """<radical>-k<kpt:3>-<spin><R|I>.[bin.]b<iorb:6> (filename_of_iorb)."""
    return "%s-k%03d-%s%s.%sb%06d" % (radical, ikpt, spin, part, "bin." if binary else "", iorb)


def _points(n, keyg):
    """(i1, i2, i3) of every point of the segments, in key order."""
    n1, n2 = n[0] + 1, n[1] + 1
    out = []
    for j0, j1 in np.asarray(keyg, np.int64).reshape(-1, 2):
        ii = j0 - 1
        i3, ii = divmod(ii, n1 * n2)
        i2, i0 = divmod(ii, n1)
        for i in range(i0, i0 + (j1 - j0) + 1):
            out.append((i, i2, i3))
    return out


def write_wave(path, psi, locreg, iorb=1, eval_=0.0, rxyz=None, binary=False):
    """Write one orbital psi ([c | f] on locreg's keys) as writeonewave does.
    locreg: wvlh.keys.Locreg (n = coarse cells per dimension)."""
    psi = np.asarray(psi, np.float64).ravel()
    nc, nf = locreg.nvctr_c, locreg.nvctr_f
    if psi.size != nc + 7 * nf:
        raise WvlhError("psi has %d values, the keys %d" % (psi.size, nc + 7 * nf))
    n = tuple(int(v) - 1 for v in locreg.n)   # maximum indices, as the reference's n1, n2, n3
    h = tuple(float(v) for v in locreg.hgrid)
    rxyz = np.zeros((0, 3)) if rxyz is None else np.asarray(rxyz, np.float64).reshape(-1, 3)
    pc, pf = _points(n, locreg.keyg_c), _points(n, locreg.keyg_f)
    fine = psi[nc:].reshape(-1, 7)
    if binary:
        with open(path, "wb") as f:
            def rec(fmt, *v):
                b = struct.pack("<" + fmt, *v)
                f.write(struct.pack("<i", len(b)) + b + struct.pack("<i", len(b)))
            rec("id", iorb, eval_)
            rec("3d", *h)
            rec("3i", *n)
            rec("i", len(rxyz))
            for r in rxyz:
                rec("3d", *r)
            rec("2i", nc, nf)
            for (i, i2, i3), t in zip(pc, psi[:nc]):
                rec("3id", i, i2, i3, t)
            for (i, i2, i3), t in zip(pf, fine):
                rec("3i7d", i, i2, i3, *t)
    else:
        lines = ["%12d %25.17E" % (iorb, eval_), "%25.17E %25.17E %25.17E" % h, "%12d%12d%12d" % n,
                 "%12d" % len(rxyz)]
        lines += ["".join(" " + fortran_e(v, 24, 17) for v in r) for r in rxyz]
        lines.append("%12d%12d" % (nc, nf))
        lines += ["%4d%4d%4d %s" % (i, i2, i3, fortran_e(t, 19, 12)) for (i, i2, i3), t in zip(pc, psi[:nc])]
        lines += ["%4d%4d%4d" % p + "".join(" " + fortran_e(v, 17, 10) for v in t) for p, t in zip(pf, fine)]
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")


_EXP3 = re.compile(r"(\d)([+-]\d{3})$")


def _num(tok):
    return float(_EXP3.sub(r"\1E\2", tok.replace("D", "E").replace("d", "e")))


def read_wave(path, binary=False):
    """Read one orbital file: dict with iorb, eval, h, n (maximum indices), rxyz,
    nvctr_c, nvctr_f, psi ([c | f]) and the points' (i1, i2, i3) (gcoord_c,
    gcoord_f), as io_read_descr + read_psi_compress."""
    if binary:
        data = open(path, "rb").read()
        pos = [0]

        def rec(fmt):
            (ln,) = struct.unpack_from("<i", data, pos[0])
            v = struct.unpack_from("<" + fmt, data, pos[0] + 4)
            if struct.calcsize("<" + fmt) != ln:
                raise WvlhError("record of %d bytes where %s was expected" % (ln, fmt))
            pos[0] += ln + 8
            return v
        iorb, ev = rec("id")
        h = rec("3d")
        n = rec("3i")
        (nat,) = rec("i")
        rxyz = np.array([rec("3d") for _ in range(nat)]).reshape(-1, 3)
        nc, nf = rec("2i")
        gc = np.zeros((nc, 3), np.int64)
        gf = np.zeros((nf, 3), np.int64)
        psi = np.zeros(nc + 7 * nf)
        for j in range(nc):
            v = rec("3id")
            gc[j] = v[:3]
            psi[j] = v[3]
        for j in range(nf):
            v = rec("3i7d")
            gf[j] = v[:3]
            psi[nc + 7 * j:nc + 7 * j + 7] = v[3:]
    else:
        lines = open(path).read().split("\n")
        it = iter(lines)

        def toks():
            return next(it).replace(",", " ").split()
        t = toks()
        iorb, ev = int(t[0]), _num(t[1])
        h = tuple(_num(v) for v in toks()[:3])
        n = tuple(int(v) for v in toks()[:3])
        nat = int(toks()[0])
        rxyz = np.array([[_num(v) for v in toks()[:3]] for _ in range(nat)]).reshape(-1, 3)
        t = toks()
        nc, nf = int(t[0]), int(t[1])
        gc = np.zeros((nc, 3), np.int64)
        gf = np.zeros((nf, 3), np.int64)
        psi = np.zeros(nc + 7 * nf)
        for j in range(nc):
            ln = next(it)   # (3(i4),1x,e19.12): fixed columns
            gc[j] = (int(ln[0:4]), int(ln[4:8]), int(ln[8:12]))
            psi[j] = _num(ln[12:].strip())
        for j in range(nf):
            ln = next(it)   # (3(i4),7(1x,e17.10))
            gf[j] = (int(ln[0:4]), int(ln[4:8]), int(ln[8:12]))
            psi[nc + 7 * j:nc + 7 * j + 7] = [_num(ln[12 + 18 * k:30 + 18 * k].strip()) for k in range(7)]
    return {"iorb": int(iorb), "eval": float(ev), "h": tuple(h), "n": tuple(int(v) for v in n), "rxyz": rxyz,
            "nvctr_c": int(nc), "nvctr_f": int(nf), "psi": psi, "gcoord_c": gc, "gcoord_f": gf}


def write_waves(radical, psi, locreg, evals=None, rxyz=None, binary=False):
    """All rows of psi (norb, ncoeff), orbitals numbered from 1 (writemywaves,
    io.f90:2760-2840, plain or binary files); returns the file names."""
    psi = np.atleast_2d(np.asarray(psi, np.float64))
    names = []
    for o in range(psi.shape[0]):
        name = wave_filename(radical, o + 1, binary)
        write_wave(name, psi[o], locreg, o + 1, 0.0 if evals is None else float(evals[o]), rxyz, binary)
        names.append(name)
    return names


def read_waves(radical, norb, locreg, binary=False):
    """The (norb, ncoeff) orbitals written by write_waves on the same keys
    (the reference reads them without reformatting when the box, grid and
    point counts agree, readonewave :298-360)."""
    out = np.zeros((norb, locreg.ncoeff))
    n = tuple(int(v) - 1 for v in locreg.n)
    for o in range(norb):
        w = read_wave(wave_filename(radical, o + 1, binary), binary)
        if w["n"] != n or w["nvctr_c"] != locreg.nvctr_c or w["nvctr_f"] != locreg.nvctr_f:
            raise WvlhError("orbital %d: the file's box or point counts differ (reformatting is not supported)"
                            % (o + 1))
        if any(abs(a - b) > 0 for a, b in zip(w["h"], locreg.hgrid)):
            raise WvlhError("orbital %d: grid spacing differs" % (o + 1))
        out[o] = w["psi"]
    return out
