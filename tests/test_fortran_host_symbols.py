"""The drop-in links against BigDFT's unchanged Fortran host: every
OpenCL-backend entry point the host calls (tests/golden/interface_ocl_symbols.txt,
made by tests/golden/make_ocl_symbols.py from bigdft/src, chiefly
interface_ocl.f90) is exported by libwvlh.so under gfortran's mangled name."""
import os
from pathlib import Path

import pytest

from wvlh._lib import exported_symbols

GOLD = Path(__file__).resolve().parent / "golden" / "interface_ocl_symbols.txt"


def listed():
    return [ln.split()[0] for ln in GOLD.read_text().splitlines() if ln.strip()]


def test_every_host_call_is_exported():
    names = listed()
    assert len(names) >= 29
    missing = sorted(set(names) - exported_symbols())
    assert not missing, "called by the Fortran host but not exported: %s" % missing


def test_symbol_list_matches_reference_sources():
    root = os.environ.get("WVLH_REFERENCE_ROOT")
    if not root or not (Path(root) / "bigdft" / "src" / "interface_ocl.f90").exists():
        pytest.skip("WVLH_REFERENCE_ROOT not set: the committed list stands")
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_ocl_symbols", GOLD.parent / "make_ocl_symbols.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    assert m.generate(root) == GOLD.read_text().splitlines()
