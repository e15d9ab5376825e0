"""Restart files in the reference's formats (writeonewave / io_read_descr /
read_psi_compress, bigdft/src/modules/io.f90:1616-1790,2639-2724; names of
filename_of_iorb, restart.f90:512-596): exact edit descriptors, record layout
of the binary form, and round trips on coarse + fine keys."""
import struct

import numpy as np
import pytest

from wvlh.keys import Locreg
from wvlh.restart import fortran_e, read_wave, read_waves, wave_filename, write_wave, write_waves


def test_fortran_e_edit_descriptor():
    assert fortran_e(-0.123456789012345, 19, 12) == "-0.123456789012E+00"
    assert fortran_e(1234.5, 19, 12) == " 0.123450000000E+04"
    assert fortran_e(0.0, 17, 10) == " 0.0000000000E+00"
    assert fortran_e(0.99999999999999, 17, 10) == " 0.1000000000E+01"
    assert fortran_e(2.5e-120, 17, 10) == " 0.2500000000-119"
    assert fortran_e(-3.0, 24, 17) == "-0.30000000000000000E+01"


def test_file_names():
    assert wave_filename("data/wavefunction", 3) == "data/wavefunction-k001-NR.b000003"
    assert wave_filename("data/wavefunction", 12, binary=True) == "data/wavefunction-k001-NR.bin.b000012"


def region(seed):
    rng = np.random.default_rng(seed)
    m = rng.random((6, 5, 7)) < 0.7
    return Locreg.from_masks(m, m & (rng.random((6, 5, 7)) < 0.5), (0, 0, 0), (0.45, 0.5, 0.55)), rng


@pytest.mark.parametrize("binary", [False, True])
def test_round_trip(tmp_path, binary):
    lr, rng = region(1)
    psi = rng.uniform(-1, 1, lr.ncoeff) * 10.0 ** rng.integers(-3, 3, lr.ncoeff)
    rxyz = rng.uniform(0, 5, (2, 3))
    p = str(tmp_path / "w")
    write_wave(p, psi, lr, iorb=4, eval_=-0.375, rxyz=rxyz, binary=binary)
    w = read_wave(p, binary)
    assert w["iorb"] == 4 and w["eval"] == -0.375 and w["n"] == (6, 4, 5)
    assert w["nvctr_c"] == lr.nvctr_c and w["nvctr_f"] == lr.nvctr_f
    assert np.allclose(w["h"], lr.hgrid, rtol=0, atol=1e-15)
    nc = lr.nvctr_c
    if binary:
        assert np.array_equal(w["psi"], psi) and np.array_equal(w["rxyz"], rxyz)
    else:   # 12 significant digits coarse, 10 fine
        assert np.all(np.abs(w["psi"][:nc] - psi[:nc]) <= 5e-12 * np.abs(psi[:nc]))
        assert np.all(np.abs(w["psi"][nc:] - psi[nc:]) <= 5e-10 * np.abs(psi[nc:]))
    # the points are the keys' grid points, in key order
    n1, n2 = lr.n[0], lr.n[1]
    lin = [i + n1 * (i2 + n2 * i3) + 1 for i, i2, i3 in w["gcoord_c"]]
    exp = np.concatenate([np.arange(a, b + 1) for a, b in lr.keyg_c])
    assert np.array_equal(lin, exp)


def test_plain_layout_and_binary_records(tmp_path):
    lr, rng = region(2)
    psi = rng.uniform(-1, 1, lr.ncoeff)
    p = str(tmp_path / "w")
    write_wave(p, psi, lr)
    lines = open(p).read().splitlines()
    first_c = lines[5]
    assert len(first_c) == 12 + 1 + 19 and first_c[12] == " "
    first_f = lines[5 + lr.nvctr_c]
    assert len(first_f) == 12 + 7 * 18
    pb = str(tmp_path / "b")
    write_wave(pb, psi, lr, binary=True)
    data = open(pb, "rb").read()
    sizes = []
    pos = 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        assert struct.unpack_from("<i", data, pos + 4 + n)[0] == n
        sizes.append(n)
        pos += n + 8
    assert sizes[:6] == [12, 24, 12, 4, 8, 20]   # no atoms: header, counts, first coarse point
    assert sizes.count(68) == lr.nvctr_f and sizes.count(20) == lr.nvctr_c


def test_waves_of_several_orbitals(tmp_path):
    lr, rng = region(3)
    psi = rng.uniform(-1, 1, (3, lr.ncoeff))
    rad = str(tmp_path / "wavefunction")
    names = write_waves(rad, psi, lr, binary=True)
    assert names[2].endswith("-k001-NR.bin.b000003")
    assert np.array_equal(read_waves(rad, 3, lr, binary=True), psi)
