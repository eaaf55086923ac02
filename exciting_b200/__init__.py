"""exciting_b200: exciting's first-variational LAPW+lo hot path on NVIDIA B200.

APW matching coefficients, Hamiltonian/overlap setup and the generalized
Hermitian eigensolve for the lowest states run as hand-written sm_100a
kernels in ``libexcfv.so`` behind the C ABI of ``include/excfv.h``.
:class:`exciting_b200.fv.FirstVariational` mirrors the reference's Fortran
interface (match, hamiltonandoverlapsetup, solvewithlapack, seceqnfv) from
Python.
"""
from .lib import load, LIB_PATH  # noqa: F401

__all__ = ["load", "LIB_PATH"]
