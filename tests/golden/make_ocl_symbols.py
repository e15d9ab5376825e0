"""Writes interface_ocl_symbols.txt: every OpenCL-backend entry point that
BigDFT's Fortran host calls, with the caller lines.

The backend's entry points are the FC_FUNC_/FC_FUNC names defined under
bigdft/src/OpenCL (C sources and headers); the host's calls are the
`call name(` statements of every Fortran source of bigdft/src except the
backend's own benchmark programs (OpenCL/conv_check*.f90,
convolutions-c/conv_check.f90).  The library must export each of them with
the trailing underscore of gfortran's name mangling.

Run from the repository root:  WVLH_REFERENCE_ROOT=<reference tree> python tests/golden/make_ocl_symbols.py
"""
import os
import re
import sys
from pathlib import Path

SKIP = {"OpenCL/conv_check.f90", "OpenCL/conv_check_fft.f90", "convolutions-c/conv_check.f90"}


def backend_names(src):
    names = set()
    for f in sorted((src / "OpenCL").glob("*")):
        if f.suffix in (".c", ".h", ".cpp"):
            names.update(m.lower() for m in re.findall(r"FC_FUNC_?\(\s*([A-Za-z0-9_]+)", f.read_text(errors="replace")))
    return names


def host_calls(src, names):
    calls = {}
    for f in sorted(src.rglob("*")):
        rel = f.relative_to(src).as_posix()
        if f.suffix.lower() not in (".f90",) or rel in SKIP:
            continue
        for i, line in enumerate(f.read_text(errors="replace").splitlines(), 1):
            code = line.split("!", 1)[0]
            for m in re.finditer(r"\bcall\s+([A-Za-z0-9_]+)", code, re.I):
                n = m.group(1).lower()
                if n in names:
                    calls.setdefault(n, []).append("%s:%d" % (rel, i))
    return calls


def generate(reference_root):
    src = Path(reference_root) / "bigdft" / "src"
    calls = host_calls(src, backend_names(src))
    out = []
    for n in sorted(calls):
        locs = calls[n]
        out.append("%s_ %s%s" % (n, " ".join(locs[:4]), " ..." if len(locs) > 4 else ""))
    return out


if __name__ == "__main__":
    root = os.environ.get("WVLH_REFERENCE_ROOT")
    if not root:
        sys.exit("set WVLH_REFERENCE_ROOT to the reference source tree")
    lines = generate(root)
    dst = Path(__file__).resolve().parent / "interface_ocl_symbols.txt"
    dst.write_text("\n".join(lines) + "\n")
    print("%d symbols -> %s" % (len(lines), dst))
