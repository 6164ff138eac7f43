"""CPU oracle of the rooftop-mom solve path: test infrastructure, never the product.

This package restates, in numpy/scipy and FP64, the MATLAB algorithm of the reference package
``+rooftopMoM`` (version 3.5.0) for the hot path: the Green's-matrix generator assembly, the
subband / embedding spectra, the split-FFT, lean split-FFT and FFT products, the circulant
preconditioners, COCG and restarted GMRES, and the plane-wave / delta-gap excitations. Every
function names the reference file and lines it follows.

Only the tests, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it, and only as the checker or the timed CPU stand-in for the MATLAB path.
The CUDA library never calls it and has no CPU fallback.

Pinning: ``tests/test_oracle_golden.py`` checks this oracle against the reference's own golden data
(``tests/data/reference.mat`` and ``tests/data/exactMoments.csv``, copied as fixtures under
``tests/golden/`` by ``tests/golden/make_golden.py``) and against the invariants of the reference's
unit tests. The reference's generators in ``reference.mat`` come from its obsolete v2 assembler and
are never compared with its current assembler, so generator parity against MATLAB itself is pinned
only through the closed-form moments and the invariant tests.
"""
