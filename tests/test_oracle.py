"""The CPU oracle is pinned against the reference's own outputs (golden fixtures)."""
import json
import os

import numpy as np
import pytest

from oracle import kp_operator as ko
from oracle import eigensolvers as oe
from oracle import post

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def test_oracle_operator_matches_reference_fixtures(operator_cases):
    assert len(operator_cases) >= 40
    for c in operator_cases:
        H = ko.confined_hamiltonian(c['shape'], c['h'], c['fields'], c['n_bands'],
                                    hole_convention=c['hole'], strain=c['strain'],
                                    include_hydrostatic=c['hydro'],
                                    interband_strain=c['interband'])
        Y = H @ c['X']
        err = np.abs(Y - c['Y']).max() / np.abs(c['Y']).max()
        assert err < 1e-13, (c['name'], err)
        assert H.nnz == c['nnz'], (c['name'], H.nnz, c['nnz'])


def test_oracle_operator_is_hermitian(operator_cases):
    for c in operator_cases[:8]:
        H = ko.confined_hamiltonian(c['shape'], c['h'], c['fields'], c['n_bands'],
                                    hole_convention=c['hole'], strain=c['strain'])
        assert oe.hermiticity_error(H) < 1e-13


def _solve_case():
    z = np.load(os.path.join(GOLDEN, 'solve_cases.npz'))
    with open(os.path.join(GOLDEN, 'solve_cases.json')) as fh:
        meta = json.load(fh)
    return z, meta


def test_oracle_small_solves_match_reference():
    """scipy LOBPCG through the oracle wrappers reproduces the reference's small solves."""
    z, meta = _solve_case()
    shape = tuple(meta['shape'])
    f8 = {k[3:]: z[k] for k in z.files if k.startswith('f8_')}
    H = ko.confined_hamiltonian(shape, float(z['h']), f8, 8, strain=True)
    assert H.nnz == meta['nnz8']
    ref = meta['interior_cb']
    E, V, info = oe.solve_interior(H, k=ref['k'], sigma=ref['sigma'], tol=ref['tol'],
                                   maxiter=ref['maxiter'])
    assert np.abs(E - np.array(ref['E'])).max() < 1e-9
    # LOBPCG iteration counts move by a few with rounding-level operator differences
    assert abs(info['iterations'] - ref['iterations']) <= 0.05 * ref['iterations']
    loc = post.localization(V, z['mask'])
    lvl, lloc, worst = post.kramers_levels(E, loc)
    assert worst < 1e-8 and len(lvl) == 2
