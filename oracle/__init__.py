"""CPU oracle for the SU(3) Wilson-fermion path (TEST INFRASTRUCTURE ONLY).

This package restates, in plain numpy complex128, the reference algorithms of
jaxQFT's Wilson-fermion hot path so that the CUDA product can be checked
against it.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline``/``--impl reference`` legs of ``bench.py`` may import it; the
product package ``jaxqft_b200`` never does.

Parity pin: ``tests/test_oracle_golden.py`` checks every function here against
golden vectors produced by running the reference's own modules
(``tests/golden/make_golden.py``) on the same inputs.
"""
