"""CPU tests: segment keys (bit-exact vs the oracle's segkeys restatement),
synthetic workloads, and the C-ABI library's exported symbols (no compute
calls: there is no GPU here)."""
import ctypes as C

import numpy as np
import pytest

from wvlh import keys as K
from wvlh import workloads as W
from wvlh._lib import LIB_PATH, exported_symbols, header_symbols


@pytest.mark.parametrize("shape,density,seed", [((5, 6, 7), 0.5, 0), ((1, 1, 1), 1.0, 1), ((3, 4, 17), 0.1, 2),
                                                 ((9, 9, 9), 0.95, 3), ((4, 4, 4), 0.0, 4)])
def test_segkeys_bit_exact(oracle, shape, density, seed):
    rng = np.random.default_rng(seed)
    m = rng.random(shape) < density
    kg, kv = K.segkeys(m)
    og, ov = oracle.segkeys(m.astype(np.uint8))
    assert np.array_equal(kg, og) and np.array_equal(kv, ov)


def test_segments_never_cross_lines():
    m = np.ones((2, 3, 4), bool)
    kg, kv = K.segkeys(m)
    assert len(kv) == 6  # one segment per (i2, i3) line
    assert np.all((kg[:, 0] - 1) // 4 == (kg[:, 1] - 1) // 4)


def test_locreg_sizes():
    lr = W.full_periodic(8)
    assert lr.nvctr_c == lr.nvctr_f == 512 and lr.ncoeff == 8 * 512
    assert lr.isf == (16, 16, 16)
    f = W.free_sphere((20, 23, 21))
    assert f.isf == (69, 75, 71) and f.fine == (54, 60, 56)
    assert 0 < f.nvctr_f < f.nvctr_c == 20 * 23 * 21


def test_gaussian_potential_shape_and_range():
    rng = np.random.default_rng(0)
    lr = W.full_periodic(10)
    V = W.gaussian_potential(lr, rng)
    assert V.shape == (20 ** 3,) and V.max() <= 0.0 and V.min() >= -8.0


def test_library_exports_every_header_symbol():
    assert LIB_PATH.exists(), "libwvlh.so must be built (make -C bigdft-suite_b200/csrc)"
    C.CDLL(str(LIB_PATH))  # loads without a GPU
    missing = header_symbols() - exported_symbols()
    assert not missing, "declared in include/wvlh.h but not exported: %s" % sorted(missing)


def test_python_symbol_lists_match_header():
    from wvlh._lib import OCL_SYMBOLS, WVLH_SYMBOLS
    assert set(OCL_SYMBOLS) | set(WVLH_SYMBOLS) == header_symbols()
