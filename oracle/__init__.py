"""CPU oracle for the meeuuw hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in vectorised numpy (plus SciPy for the sparse direct
solves the reference itself uses), the reference algorithms of cedrict/meeuuw
that the CUDA library replaces.  Every function cites the reference file:line it
follows.  It is the checker: only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.  The
product package ``meeuuw_b200`` never imports it and has no CPU fallback.

Parity of this oracle is pinned against golden vectors produced by importing
the reference's own Numba functions (``tests/golden/make_golden.py``, run in a
container that has the reference checkout) and committed as ``.npz`` fixtures.
"""
