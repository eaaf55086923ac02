"""CPU oracle for the first-variational LAPW+lo hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``exciting_b200`` package imports
this package: it is used by ``tests/``, by ``__graft_entry__.smoke()`` as the
checker, and by ``bench.py`` for the timed CPU baseline / reference arm.

It restates, in NumPy, the reference's own algorithm for each routine on the
path (each function cites the Fortran file and lines it follows) and calls
LAPACK's ZHEGVX through SciPy with exactly the reference's arguments
(``src/src_eigensystem/modfvsystem.f90:691-693``: itype 1, 'V', 'I', 'U',
il=1, iu=nstfv, abstol=evaltol, lwork=2n).

Pinning.  The reference is Fortran and cannot be compiled here (no Fortran
compiler), and no reference test pins the setup or the eigensolve in
isolation.  The pieces that the reference's tests do pin are checked:
``genylm``/``sbessel`` against the plane-wave (Rayleigh) expansion used by
``src/math/sh_product_test.f90:136-175``, plus closed forms of j_l and Y_lm.
The eigensolve is LAPACK's own ZHEGVX (the routine the reference links).
The setup restatement itself is unpinned by reference fixtures; it is checked
against independent formulations (A^H aa A built from the definition, the
interstitial matrix built from the Fourier coefficients directly).

``two_stage`` restates the published two-stage Householder tridiagonal
reduction (dense -> band -> tridiagonal) with explicit reflectors, the
checker for a GPU reduction that follows the same reflector order.
"""
