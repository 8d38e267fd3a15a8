"""CPU oracle for the ART hot path -- TEST INFRASTRUCTURE ONLY.

A restatement of the reference's CPU algorithms (numpy/scipy, the same
third-party numerics the reference calls), used by ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg to check and
time the B200 kernels.  Nothing in the ``art`` package imports it; the
product path never routes through it.

Pinning: every restated function is checked against fixtures generated from
the reference implementation itself (``tests/golden/make_golden.py`` imports
the reference package under the name ``art_ref`` and records its outputs).
The hit-and-run KS-uniformity/autocorrelation targets are statistical and
have no reference golden values (the reference asserts none).
"""
