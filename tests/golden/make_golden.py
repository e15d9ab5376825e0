"""Generate the committed golden vectors of tests/golden.

magicfilter_ref.npz — outputs of the REFERENCE's own C magic filter
(bigdft/src/convolutions-c/MagicFilter_sse.c, magicfilter1d_naive_ and
magicfilter1d_t_naive_), compiled by oracle/Makefile into oracle/_ref from the
reference tree, on a seeded input.  These pin the oracle's magic filter where
the reference tree is absent (e.g. on the GPU machine).

locham_small.npz — small local-Hamiltonian cases computed by the CPU oracle
(regression vectors for the GPU parity tests; they are not reference outputs).

Run from the repository root:  python tests/golden/make_golden.py
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle as O  # noqa: E402


def magicfilter():
    R = O.ref_magicfilter()
    if R is None:
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    rng = np.random.default_rng(1234)
    n, ndat = 20, 6
    out = {"n": n, "ndat": ndat}
    for key, fn in (("n", "magicfilter1d_naive_"), ("t", "magicfilter1d_t_naive_")):
        x = rng.uniform(-1, 1, n * ndat)
        y = np.zeros(n * ndat)
        getattr(R, fn)(C.byref(C.c_uint(n)), C.byref(C.c_uint(ndat)), x, y)
        out["x_" + key], out["y_" + key] = x, y
    np.savez(Path(__file__).with_name("magicfilter_ref.npz"), **out)


def locham_small():
    rng = np.random.default_rng(99)
    out = {}
    cases = [("per", (8, 9, 10), (1, 1, 1)), ("free", (6, 7, 5), (0, 0, 0)), ("surf", (8, 6, 8), (1, 0, 1))]
    for name, N, per in cases:
        mc = np.ones(N[::-1], np.uint8)
        mf = (rng.random(N[::-1]) < 0.5).astype(np.uint8)
        d = O.desc_from_masks(mc, mf, per)
        pc, pf = rng.uniform(-1, 1, d.nvctr_c), rng.uniform(-1, 1, 7 * d.nvctr_f)
        pot = rng.uniform(-1, 0, int(np.prod(d.I)))
        h = (0.45, 0.4, 0.5)
        hc, hf, ek, ep = O.locham(d, h, pc, pf, pot)
        out.update({name + "_mf": mf, name + "_psi": np.concatenate([pc, pf]), name + "_pot": pot,
                    name + "_hpsi": np.concatenate([hc, hf]), name + "_e": np.array([ek, ep])})
    np.savez_compressed(Path(__file__).with_name("locham_small.npz"), **out)


if __name__ == "__main__":
    magicfilter()
    locham_small()
    print("golden vectors written")
