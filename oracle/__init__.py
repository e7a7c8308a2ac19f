"""CPU oracle for funlbm's per-step lattice-Boltzmann path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this package, and only as the checker
(or as the timed CPU baseline).  The product path (``funlbm_b200``) never imports
it: there is no CPU fallback.

The oracle is pinned against golden vectors produced by running the reference
itself (funlbm 1.2.0) in the build container; see ``tests/golden/make_golden.py``
and ``tests/test_oracle_golden.py``.
"""
