"""The benchmark's counting rule (bench.checked_pairs): an eigenpair counts only if it is within
1e-6 eV of the reference's own eigenvalue, its Kramers partner within 1e-7 eV, and its relative
residual ||Hv - Ev|| / ||H||_2 at most 1e-8. Checked on the reference's own b = 10 nm solve."""
import json
import os

import numpy as np

import bench

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _ref():
    with open(os.path.join(GOLDEN, 'fig4_b10.json')) as fh:
        return json.load(fh)


def test_reference_levels_with_small_residuals_all_count():
    ref = _ref()
    E = np.array(ref['cb']['E'])
    res = np.full(8, 1e-9)
    n, dE, rel, split = bench.checked_pairs(E, res, ref['cb'], ref['H_norm2'])
    assert n == 8 and dE == 0.0 and split < 1e-12


def test_each_check_removes_pairs():
    ref = _ref()
    E = np.array(ref['cb']['E'])
    hn = ref['H_norm2']
    res = np.full(8, 1e-9)
    # the reference's own residuals (tol 1e-7) exceed 1e-8 relative for some of its states
    n, _, rel, _ = bench.checked_pairs(E, np.array(ref['cb']['residuals']), ref['cb'], hn)
    assert n < 8 and rel > 1e-8
    # one level shifted by 2e-6 eV: both of its states leave the count
    E2 = E.copy()
    E2[2:4] += 2e-6
    assert bench.checked_pairs(E2, res, ref['cb'], hn)[0] == 6
    # a split Kramers pair (one partner moved by 5e-7 eV, still within 1e-6 of the reference)
    E3 = E.copy()
    E3[5] += 5e-7
    assert bench.checked_pairs(E3, res, ref['cb'], hn)[0] == 6
    # order does not matter
    p = np.random.default_rng(0).permutation(8)
    assert bench.checked_pairs(E[p], res[p], ref['cb'], hn)[0] == 8
