"""CPU oracle for the LH82 anelastic step — TEST INFRASTRUCTURE ONLY.

This package restates, in plain NumPy, the reference algorithm of Oracle V8's
dynamical-core step (justingwatford-dev/Oraclev8, ``oracle_v8/solver``).  It is
the checker the CUDA path is compared against: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product package ``oraclev8_b200`` never imports, calls or links
anything here, and has no CPU fallback.

Parity of this restatement is pinned by ``tests/test_oracle_golden.py`` against
fixtures produced by running the unmodified reference (see
``tests/golden/make_golden.py``), plus the scalar known answers of the
reference's own tests.
"""
