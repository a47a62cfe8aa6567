"""CPU oracle for the classicalDFT F[rho] / dF/drho hot path (FP64, NumPy/SciPy).

TEST INFRASTRUCTURE ONLY.  This package is a restatement of the reference
library's algorithm for the checker: the tests under ``tests/``, the
``smoke()`` self-check in ``__graft_entry__`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` import it.  The product
(``classicaldft_b200`` and its CUDA library) never imports, calls or links
anything here, and there is no CPU fallback in the product.

Provenance.  The reference (migduroli/classicalDFT v3.0.0) cannot be compiled
in this environment: its hot path needs Armadillo, FFTW3, GSL and autodiff,
none of which is installed, and its build fetches dependencies over the
network.  Every function here cites the reference file:line it restates.
Parity of this restatement is pinned by the reference's own known-answer
tests (analytic sum rules, bulk limits, PY/CS identities, FD derivative
checks; see ``tests/test_oracle_*.py``) and by an independent second source:
the legacy formulas of ``legacy/classicaldft.hpp`` restated in
``oracle/legacy.py``.

Third-party arithmetic on the path and how it is restated:
  * FFTW3 (version unpinned; Debian trixie ``libfftw3-dev``): r2c / unnormalised
    c2r of ``src/math/fourier.cpp:97-103``.  Restated with ``scipy.fft``
    (pocketfft); c2r of non-Hermitian input follows FFTW's rank>=2 c2r
    semantics (complex transforms over x, y, then a 1-D c2r over z that drops
    the imaginary parts of the kz=0 and kz=Nz/2 planes), which is exactly the
    Hermitian projection ``grid.hermitian_project``.
  * autodiff v1.1.2 (forward duals, ``include/dft/math/autodiff.hpp``):
    f'(eta) of ``models.hpp:59-61``.  Restated as closed-form derivatives of
    the same expressions (``oracle/fmt.py``), checked against central finite
    differences as the reference's own tests do.
  * GSL QAGS (``include/dft/math/integration.hpp``): setup-time integrals
    (hard-sphere diameter, van der Waals integral).  Restated with
    ``scipy.integrate.quad`` (QUADPACK QAGS, the same algorithm).
  * Armadillo ``eig_sym`` on 3x3 (``saddle_point.hpp:253``): ``numpy.linalg.eigh``.
"""
