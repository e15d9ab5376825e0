"""Writes opencl_kernels.npz: outputs of the reference's OpenCL periodic
wavelet synthesis and analysis kernels (bigdft/src/OpenCL/Wavelet_Generator.cpp:
syn1dKernel_d, ana1dKernel_d) and fine-grid kinetic kernel
(bigdft/src/OpenCL/Kinetic_Generator.cpp: kinetic1dKernel_d) and free-BC
magic filters (bigdft/src/OpenCL/MagicFilter_Generator.cpp), evaluated on
seeded lines.

The kernels exist only as source text that the generator pastes into an
OpenCL program; there is no OpenCL runtime here.  This script reads the
generator's scalar filter macros and replays their multiply-add statements in
their own order, with the indexing of the kernels that use them:

  * analysis (`filter(ci,di,tmp)` in generate_ana_filter, used by
    generate_ana1dKernel): for coarse output i of a line of 2n fine points,
    tmp[m] = psi[(2 i - 7 + m) mod 2n]; out[i] = ci, out[i + n] = di;
  * synthesis (`filter(tmp1,tmp2)` in generate_syn_filter, used by
    generate_syn1dKernel): tmp1 points at s[i - 4] and tmp2 at w[i - 4] of the
    line's two halves (s = psi[0:n], w = psi[n:2n], periodic in the coarse
    index); the macro starts tmp1b = tmp1, tmp2b = tmp2 + 8 and walks them
    with ++ / --; out[2 i] = se, out[2 i + 1] = so;
  * free-BC synthesis (`filter_grow(tmp1,tmp2)`, used by
    generate_syngrow1dKernel): Nc coarse points grow to Nc + 7 output pairs,
    tmp1 / tmp2 at s[i - 7] / w[i - 7] (zero outside), out[2 i] = so,
    out[2 i + 1] = se; free-BC analysis (the analysis macro in
    generate_anashrink1dKernel): tmp[m] = y[2 i + m] of 2 Nc + 14 points;
  * free-BC magic filter (`filter(tmp)` / `filter_reverse(tmp)` of
    MagicFilter_Generator.cpp with its FILT* values, used by
    generate_magicfiltergrow1dKernel / generate_magicfiltershrink1dKernel):
    growing, tmp[k] = x[i - 15 + k] (zero outside); shrinking, tmp[k] = y[i + k];
  * kinetic (`filter1(tt,tmp)` in generate_filters, with the FILT1_* values
    of generate_header, used by generate_kinetic1dKernel): for fine point i of
    a line of n points, tmp[m] = x[(i + m) mod n]; the kernel writes
    y_in + scale * conv, of which the file keeps conv.

`mad(a, b, c)` is evaluated as a * b + c in FP64.  The file holds, per line
length n, the input line and the two kernels' outputs.

Run from the repository root:
  WVLH_REFERENCE_ROOT=<reference tree> python tests/golden/make_opencl_kernels.py
"""
import os
import re
import sys
from pathlib import Path

import numpy as np

NUM = r"([-+]?[0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?)"


def macro(text, head):
    """Body of the first `#define <head>` macro of the generator's text."""
    i = text.index("#define " + head)
    j = text.find("#define", i + 1)
    k = text.find('";', i)
    end = min(x for x in (j, k) if x > 0)
    return text[i + len("#define " + head):end]


def ana_program(text):
    body = macro(text, "filter(ci,di,tmp)")
    prog = [(v, int(m), float(c)) for v, m, c, v2 in
            re.findall(r"(ci|di)\s*=\s*mad\(\s*tmp\[\s*(\d+)\s*\]\s*,\s*" + NUM + r"\s*,\s*(ci|di)\s*\)", body)]
    assert len(prog) == 32, len(prog)
    return prog


def syn_program(text, head="filter(tmp1,tmp2)"):
    body = macro(text, head)
    st = re.findall(r"(se|so)\s*=\s*mad\(\s*\*\s*(tmp1b|tmp2b)\s*(\+\+|--)?\s*,\s*" + NUM + r"\s*,\s*(se|so)\s*\)", body)
    init = dict(re.findall(r"(tmp[12]b)\s*=\s*tmp[12]\s*(?:\+\s*(\d+))?\s*;", body.replace("__local double *", "")))
    start = {"tmp1b": int(init.get("tmp1b") or 0), "tmp2b": int(init.get("tmp2b") or 0)}
    prog = [(v, p, inc, float(c)) for v, p, inc, c, v2 in st]
    assert len(prog) == 32 and set(init) == {"tmp1b", "tmp2b"}, (len(prog), init)
    return prog, start


def mf_program(text, head):
    """Tap values of a magic-filter macro (`filter(tmp)` or `filter_reverse(tmp)`
    of MagicFilter_Generator.cpp) in the order its statements apply them to
    tmp[0], tmp[1], ..."""
    filt = {int(k): float(v) for k, v in re.findall(r"#define FILT(\d+)\s+" + NUM, text)}
    body = macro(text, head)
    order = [int(k) for k in re.findall(r"tt\s*=\s*mad\(\s*\*tmp\+\+\s*,\s*FILT(\d+)\s*,\s*tt\s*\)", body)]
    assert len(order) == 16 and len(filt) == 16, (len(order), len(filt))
    return [filt[k] for k in order]


def mfgrow_line(taps, x):
    """magicfiltergrow1dKernel_d: Lf inputs (zero outside), Lf + 15 outputs;
    tmp[k] = x[i - 15 + k]."""
    lf = len(x)
    out = np.zeros(lf + 15)
    for i in range(lf + 15):
        tt = 0.0
        for k, c in enumerate(taps):
            j = i - 15 + k
            tt = (x[j] if 0 <= j < lf else 0.0) * c + tt
        out[i] = tt
    return out


def mfshrink_line(taps, y):
    """magicfiltershrink1dKernel_d: Lf + 15 inputs, Lf outputs; tmp[k] = y[i + k]."""
    lf = len(y) - 15
    out = np.zeros(lf)
    for i in range(lf):
        tt = 0.0
        for k, c in enumerate(taps):
            tt = y[i + k] * c + tt
        out[i] = tt
    return out


def kin_program(text):
    filt = {int(k): float(v) for k, v in re.findall(r"#define FILT1_(\d+)\s+" + NUM, text)}
    body = macro(text, "filter1(tt,tmp)")
    prog = []
    for a, b, k in re.findall(r"tt\s*=\s*mad\(\s*tmp\[\s*(-?\d+)\s*\](?:\s*\+\s*tmp\[\s*(-?\d+)\s*\])?\s*,"
                              r"\s*FILT1_(\d+)\s*,\s*tt\s*\)", body):
        prog.append((int(a), None if b == "" else int(b), filt[int(k)]))
    assert len(prog) == 15 and len(filt) == 15, (len(prog), len(filt))
    return prog


def kin_line(prog, x):
    n = len(x)
    out = np.zeros(n)
    for i in range(n):
        tt = 0.0
        for a, b, c in prog:
            v = x[(i + a) % n] if b is None else x[(i + a) % n] + x[(i + b) % n]
            tt = v * c + tt
        out[i] = tt
    return out


def ana_line(prog, x):
    n = len(x) // 2
    out = np.zeros(2 * n)
    for i in range(n):
        tmp = [x[(2 * i - 7 + m) % (2 * n)] for m in range(16)]
        acc = {"ci": 0.0, "di": 0.0}
        for v, m, c in prog:
            acc[v] = tmp[m] * c + acc[v]
        out[i], out[i + n] = acc["ci"], acc["di"]
    return out


def syn_line(prog, start, x):
    n = len(x) // 2
    s, w = x[:n], x[n:]
    out = np.zeros(2 * n)
    for i in range(n):
        pos = {"tmp1b": start["tmp1b"], "tmp2b": start["tmp2b"]}
        src = {"tmp1b": s, "tmp2b": w}
        acc = {"se": 0.0, "so": 0.0}
        for v, p, inc, c in prog:
            acc[v] = src[p][(i - 4 + pos[p]) % n] * c + acc[v]
            pos[p] += 1 if inc == "++" else -1 if inc == "--" else 0
        out[2 * i], out[2 * i + 1] = acc["se"], acc["so"]
    return out


def syngrow_line(prog, start, x):
    """syngrow1dKernel_d: coarse inputs s, w of Nc points each (zero outside),
    n = Nc + 7 output pairs; tmp1 at s[i - 7], tmp2 at w[i - 7]."""
    nc = len(x) // 2
    s, w = x[:nc], x[nc:]
    n = nc + 7
    out = np.zeros(2 * n)
    for i in range(n):
        pos = {"tmp1b": start["tmp1b"], "tmp2b": start["tmp2b"]}
        src = {"tmp1b": s, "tmp2b": w}
        acc = {"se": 0.0, "so": 0.0}
        for v, p, inc, c in prog:
            k = i - 7 + pos[p]
            val = src[p][k] if 0 <= k < nc else 0.0
            acc[v] = val * c + acc[v]
            pos[p] += 1 if inc == "++" else -1 if inc == "--" else 0
        out[2 * i], out[2 * i + 1] = acc["so"], acc["se"]
    return out


def anashrink_line(prog, y):
    """anashrink1dKernel_d: 2 Nc + 14 fine inputs, Nc coarse outputs;
    tmp[m] = y[2 i + m]."""
    nc = (len(y) - 14) // 2
    out = np.zeros(2 * nc)
    for i in range(nc):
        acc = {"ci": 0.0, "di": 0.0}
        for v, m, c in prog:
            acc[v] = y[2 * i + m] * c + acc[v]
        out[i], out[i + nc] = acc["ci"], acc["di"]
    return out


def main():
    root = os.environ.get("WVLH_REFERENCE_ROOT") or (sys.argv[1] if len(sys.argv) > 1 else None)
    if not root:
        sys.exit("set WVLH_REFERENCE_ROOT to the reference tree")
    text = (Path(root) / "bigdft/src/OpenCL/Wavelet_Generator.cpp").read_text()
    ana = ana_program(text)
    syn, start = syn_program(text)
    kin = kin_program((Path(root) / "bigdft/src/OpenCL/Kinetic_Generator.cpp").read_text())
    grow, gstart = syn_program(text, "filter_grow(tmp1,tmp2)")
    mtext = (Path(root) / "bigdft/src/OpenCL/MagicFilter_Generator.cpp").read_text()
    mf_fwd, mf_rev = mf_program(mtext, "filter(tmp)"), mf_program(mtext, "filter_reverse(tmp)")
    rng = np.random.default_rng(2024)
    out = {}
    for n in (8, 9, 13, 16, 24):
        x = rng.uniform(-1, 1, 2 * n)
        out["x_%d" % n] = x
        out["ana_%d" % n] = ana_line(ana, x)
        out["syn_%d" % n] = syn_line(syn, start, x)
        out["kin_%d" % n] = kin_line(kin, x)   # on the 2n fine points of the same line
        out["grow_%d" % n] = syngrow_line(grow, gstart, x)   # free BC: n coarse points grow to 2n + 14
        yg = rng.uniform(-1, 1, 2 * n + 14)
        out["yg_%d" % n] = yg
        out["shrink_%d" % n] = anashrink_line(ana, yg)
        out["mfgrow_%d" % n] = mfgrow_line(mf_fwd, x)        # 2n fine points grow by 15
        ym = rng.uniform(-1, 1, 2 * n + 15)
        out["ym_%d" % n] = ym
        out["mfshrink_%d" % n] = mfshrink_line(mf_rev, ym)
    dst = Path(__file__).resolve().parent / "opencl_kernels.npz"
    np.savez(dst, **out)
    print("wrote", dst, "syn start", start)


if __name__ == "__main__":
    main()
