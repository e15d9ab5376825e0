"""wvlh — B200-native Daubechies-16 wavelet local Hamiltonian (BigDFT's locham hot path).

Python host side of the library.  Everything here drives ``libwvlh.so`` (CUDA
kernels for sm_100a behind a C ABI, see ``include/wvlh.h``); there is no CPU
fallback: importing works on any machine, but every compute call raises if the
shared library or a CUDA device is missing.

* :mod:`wvlh.keys` — segment keys from a logical grid (the reference's
  ``num_segkeys``/``segkeys``, ``bigdft/src/locregs/initlocregs.f90:1573,1633``).
* :mod:`wvlh.batch` — batched local Hamiltonian over many orbitals and
  localisation regions (FP32 / FP64 fused, FP64 plain per-pass).
* :mod:`wvlh.ocl` — the drop-in ``ocl_*`` entry points that BigDFT's
  ``interface_ocl.f90`` calls, and a Python mirror of its
  ``local_hamiltonian_OCL`` / ``local_partial_density_OCL`` /
  ``preconditionall_OCL`` drivers.
* :mod:`wvlh.workloads` — seeded synthetic inputs with the shapes of the
  benchmark configurations.
"""
from ._lib import LIB_PATH, WvlhError, lib  # noqa: F401
from .keys import segkeys, Locreg  # noqa: F401
