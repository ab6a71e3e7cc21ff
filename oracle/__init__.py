"""CPU oracle for the hex8 linear-elastic path -- TEST INFRASTRUCTURE ONLY.

This package is a plain NumPy/SciPy restatement of abhi2k16/computation-suite's
``fea_engine`` algorithms for the hex8 assembly + Jacobi-PCG static path (plus the
SIMP compliance sensitivity and the POD singular values).  Every function cites
the reference file:line it follows.

It exists to CHECK the CUDA library, never to stand in for it:
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import it.  The product package (``feab200``) never imports it and fails
loudly when its CUDA library is missing.

Parity pin: ``tests/golden/`` holds vectors generated by running the reference
itself (``tests/golden/make_golden.py``); ``tests/test_oracle_golden.py`` checks
this restatement against them.
"""
from .fea_oracle import *  # noqa: F401,F403
