"""CPU oracle for the cross-sectional analysis path (TEST INFRASTRUCTURE ONLY).

Nothing in the product imports this package.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may use it, and only as the checker or as the timed CPU
baseline -- never as the thing measured for the GPU path.

Parity pinning: ``fc_oracle`` is checked against golden vectors produced by the
reference's own CPU path (``fc/_cpu_core.py``) and by its frozen fixtures
(``benchmark_corpus/parity_anchors_v1``, ``tests/fixtures/corr_corpus_v1``);
see ``tests/golden/make_golden.py`` and ``tests/test_oracle_pins.py``.
"""
