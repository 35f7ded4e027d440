"""CPU oracle for the eight-band k.p eigensolve path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product path (the `qd3dsolver_b200` package and its CUDA library) imports,
links or calls this package. Only `tests/`, `__graft_entry__.smoke()` and the CPU-baseline
legs of `bench.py` use it, and only as the checker or as the timed CPU baseline.

Contents
--------
kp_operator  -- NumPy/SciPy restatement of qd3Dsolver's discretised Pryor eight-band operator
                (kp_confined.py:58-183, kp_pryor.py:74-153, 216-301, 363-466) as a CSR matrix.
eigensolvers -- restatement of eigensolvers.py's folded-spectrum / extremal LOBPCG wrappers
                (eigensolvers.py:76-135, 200-268, 301-386) around the third-party
                scipy.sparse.linalg.lobpcg the reference calls.
post         -- localisation and Kramers pairing (pryor_fig4.py:179-193, 222-236).

Parity pins: the operator is checked against H @ X fixtures generated by the reference itself
(tests/golden/make_golden.py), and the solver wrappers against the reference's own solves on
small grids and on the seven Fig-4 pyramids of pryor_fig4.sweep with the reference's own FD-strain
fields (tests/golden/make_fig4_golden.py). On the 48x48x36 pyramid the reference's folded solve
does not converge (spurious finite-difference band, tests/test_spurious_band.py); its first
LOBPCG iterations are the fixture there (tests/golden/make_config1_golden.py).
"""
