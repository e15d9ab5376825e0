"""Regenerate ``wvl_filters.h`` from the reference's own source files.

The Daubechies-16 two-scale coefficients, the magic filter, the 29-tap
second-derivative filters and the preconditioner diagonal constants must be
bit-identical to the ones the reference compiles, so they are parsed out of
the reference sources instead of being retyped:

* DB16 analysis ``ch/cg(-7:8)``: ``bigdft/src/orbitals/convolut_simple_per.f90:22-39``
  (``ana_rot_per``); synthesis uses the same numbers shifted to ``(-8:9)``
  (``:70-87``).
* magic filter ``fil(-8:7)``: ``convolut_simple_per.f90:214-230`` (``convrot_n_per``);
  the transposed filter ``(-7:8)`` at ``:260-276`` is its mirror image.
* kinetic ``fil(0:14)`` (``<phi|D2|phi>``): ``convolut_simple_per.f90:396-410``.
* wavelet-basis kinetic blocks ``c`` (``<phi|D2|psi>``) and ``e``
  (``<psi|D2|psi>``): ``bigdft/src/orbitals/convolut_ib_optim.f90:987-1046``
  (``ConvolkineticT``); ``a`` equals the kinetic ``fil`` and ``b(i)=c(-i)``.
* preconditioner diagonal ``A2``/``B2``: ``bigdft/src/OpenCL/Uncompress.c:377-378``.
* the 89-term Gaussian expansion of 1/r that the free-boundary Poisson kernel
  is built from (exponents ``p`` and weights ``w``, range [1e-9, 1]):
  ``psolver/src/Build_Kernel.f90:1679-1873`` (``gequad``).
* the Gaussian fits of the wire-BC kernel (log r at zero frequency: ``p1``,
  ``w1``; K0(r) otherwise: ``p2``, ``w2``; the first 144 of 150 are used):
  ``psolver/src/gaussfit_wires.inc``.

Run ``python gen_filters.py <reference source tree>`` to rewrite the header; the
generated header is committed so that the build never needs the reference.
"""
import re
import sys
from pathlib import Path

NUM = r"[-+]?\d*\.?\d+(?:[eEdD][-+]?\d+)?"


def _fortran_numbers(text):
    out = []
    for m in re.finditer(r"(" + NUM + r")(?:_wp|_gp)?", text):
        s = m.group(1).replace("d", "e").replace("D", "e")
        out.append(s)
    return out


def _data_block(src, name, start_line):
    """Return the numbers of the first ``data <name> / ... /`` after start_line."""
    lines = src.splitlines()[start_line - 1:]
    text = "\n".join(lines)
    m = re.search(r"data\s+" + name + r"\s*/(.*?)/", text, re.S | re.I)
    if not m:
        raise ValueError("data block %s not found" % name)
    body = re.sub(r"&", " ", m.group(1))
    return _fortran_numbers(body)


def _indexed(src, name, lo, hi, start_line):
    """Collect ``name(i)= value`` assignments (first occurrence after start_line)."""
    lines = src.splitlines()[start_line - 1:]
    vals = {}
    pat = re.compile(r"^\s*" + name + r"\(\s*(-?\d+)\s*(?:,\s*:\s*)?\)\s*=\s*(" + NUM + r")", re.I)
    for ln in lines:
        m = pat.match(ln)
        if m:
            i = int(m.group(1))
            if lo <= i <= hi and i not in vals:
                vals[i] = m.group(2).replace("d", "e").replace("D", "e")
        if len(vals) == hi - lo + 1:
            break
    if len(vals) != hi - lo + 1:
        raise ValueError("incomplete filter %s: %d of %d" % (name, len(vals), hi - lo + 1))
    return [vals[i] for i in range(lo, hi + 1)]


def parse(ref_root):
    src_dir = Path(ref_root) / "bigdft" / "src"
    simple = (src_dir / "orbitals" / "convolut_simple_per.f90").read_text()
    ib = (src_dir / "orbitals" / "convolut_ib_optim.f90").read_text()
    unc = (src_dir / "OpenCL" / "Uncompress.c").read_text()

    ana_line = simple.splitlines().index(next(l for l in simple.splitlines() if "subroutine ana_rot_per" in l)) + 1
    ch = _data_block(simple, "ch", ana_line)
    cg = _data_block(simple, "cg", ana_line)
    assert len(ch) == 16 and len(cg) == 16
    mf_line = next(i for i, l in enumerate(simple.splitlines(), 1) if "subroutine convrot_n_per" in l)
    mf = _fortran_numbers(re.search(r"DATA\s+fil\s*/(.*?)/", "\n".join(simple.splitlines()[mf_line - 1:]), re.S).group(1).replace("&", " "))
    assert len(mf) == 16
    kin_line = next(i for i, l in enumerate(simple.splitlines(), 1) if "subroutine convolut_kinetic_per_T" in l)
    kin = _indexed(simple, "fil", 0, 14, kin_line)
    ckt_line = next(i for i, l in enumerate(ib.splitlines(), 1) if "subroutine ConvolkineticT" in l)
    cwav = _indexed(ib, "c", -14, 14, ckt_line)
    ewav = _indexed(ib, "e", 0, 14, ckt_line)
    a2 = re.search(r"#define\s+A2\s+(" + NUM + ")", unc).group(1)
    b2 = re.search(r"#define\s+B2\s+(" + NUM + ")", unc).group(1)
    bk = (Path(ref_root) / "psolver" / "src" / "Build_Kernel.f90").read_text()
    gq_line = next(i for i, l in enumerate(bk.splitlines(), 1) if re.match(r"\s*subroutine gequad\(", l))
    gq_p = _indexed(bk, "p", 1, 89, gq_line)
    gq_w = _indexed(bk, "w", 1, 89, gq_line)
    gw = (Path(ref_root) / "psolver" / "src" / "gaussfit_wires.inc").read_text()
    wires = {}
    for name in ("p1", "w1", "p2", "w2"):
        body = re.search(r"^\s*" + name + r"\s*=\s*\(/(.*?)/\)", gw, re.S | re.M).group(1)
        vals = [v.replace("d", "e").replace("D", "e") for v in
                re.findall(NUM, re.sub(r"_dp", "", body.replace("&", " ")))]
        assert len(vals) == 150, (name, len(vals))
        wires[name] = vals
    return dict(ch=ch, cg=cg, mf=mf, kin=kin, cwav=cwav, ewav=ewav, a2=a2, b2=b2, gq_p=gq_p, gq_w=gq_w,
                wires=wires)


def render(f):
    def arr(name, vals, comment, at=True):
        body = ", \\\n".join("    %s" % v for v in vals)
        out = ("/* %s */\n#define %s_INIT { \\\n%s}\nstatic const double %s[%d] = %s_INIT;\n"
               % (comment, name, body, name, len(vals), name))
        if at:
            # NAME_AT(i): the i-th tap as a constant expression (folds to an
            # immediate when i is a compile-time constant)
            expr = "".join("(i) == %d ? (%s) : " % (k, v) for k, v in enumerate(vals)) + "0.0"
            out += "#define %s_AT(i) (%s)\n" % (name, expr)
        return out

    parts = [
        "/* Generated by gen_filters.py from the reference sources; do not edit. */",
        "#pragma once",
        "",
        arr("WVL_CH", f["ch"], "DB16 low-pass ch(-7..8): convolut_simple_per.f90:22-30 (index l+7)"),
        arr("WVL_CG", f["cg"], "DB16 high-pass cg(-7..8): convolut_simple_per.f90:31-39 (index l+7)"),
        arr("WVL_MF", f["mf"], "magic filter fil(-8..7): convolut_simple_per.f90:214-230 (index l+8)"),
        arr("WVL_KIN", f["kin"], "second-derivative <phi|D2|phi> fil(0..14): convolut_simple_per.f90:396-410"),
        arr("WVL_KIN_C", f["cwav"], "<phi|D2|psi> c(-14..14): convolut_ib_optim.f90:987-1015 (index l+14)"),
        arr("WVL_KIN_E", f["ewav"], "<psi|D2|psi> e(0..14): convolut_ib_optim.f90:1021-1035"),
        "/* preconditioner diagonal constants: OpenCL/Uncompress.c:377-378 */",
        "#define WVL_A2 %s" % f["a2"],
        "#define WVL_B2 %s" % f["b2"],
        arr("WVL_GQ_P", f["gq_p"], "1/r = sum w(i) exp(-p(i) r^2), r in [1e-9, 1]: exponents p(1..89), "
            "psolver/src/Build_Kernel.f90:1689-1777 (gequad)", at=False),
        arr("WVL_GQ_W", f["gq_w"], "weights w(1..89): Build_Kernel.f90:1779-1867", at=False),
        arr("WVL_WIRE_P1", f["wires"]["p1"], "log r = sum w1 exp(-p1 r^2) (wire BC, zero frequency): exponents, "
            "psolver/src/gaussfit_wires.inc (p1)", at=False),
        arr("WVL_WIRE_W1", f["wires"]["w1"], "weights w1: gaussfit_wires.inc", at=False),
        arr("WVL_WIRE_P2", f["wires"]["p2"], "K0(r) = sum w2 exp(-p2 r^2) (wire BC): exponents, gaussfit_wires.inc",
            at=False),
        arr("WVL_WIRE_W2", f["wires"]["w2"], "weights w2: gaussfit_wires.inc", at=False),
        "",
    ]
    return "\n".join(parts)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python gen_filters.py <reference source tree>")
    ref = sys.argv[1]
    out = Path(__file__).with_name("wvl_filters.h")
    out.write_text(render(parse(ref)))
    print("wrote", out)
