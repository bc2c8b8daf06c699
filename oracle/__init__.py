"""CPU oracle (test infrastructure only).

A NumPy float64 restatement of the reference's solve arithmetic, used by
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` as the checker.  Nothing in the ``pylcm_b200`` package imports
this directory; the product path never calls it.

Parity is pinned against the reference's own stored float64 outputs
(``tests/data/regression_tests/solution.pkl`` and
``tests/data/processes/solution_*.pkl`` of the reference project, committed
here as ``tests/golden/*.npz`` by ``tests/golden/make_golden.py``).
"""
