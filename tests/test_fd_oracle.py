"""The CPU restatement of the inhomogeneous FD elasticity solve (oracle/elasticity_fd.py) against
the reference's own solve_strain_fd: the small cases of tests/golden/make_fd_golden.py and the
FD strain of the b = 6 nm Fig-4 environment (tests/golden/make_fig4_golden.py)."""
import json
import os

import numpy as np

from oracle import elasticity_fd as ofd

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
STRAIN = ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')


def _cases():
    with open(os.path.join(GOLDEN, 'fd_strain_cases.json')) as fh:
        meta = json.load(fh)
    return meta, np.load(os.path.join(GOLDEN, 'fd_strain_cases.npz'))


def test_oracle_fd_strain_matches_reference_cases():
    meta, arr = _cases()
    for c in meta['cases']:
        t = c['tag']
        strain, info = ofd.solve_strain_fd(arr[f'{t}_mask'], c['eps_star'], tuple(c['C_dot']),
                                           tuple(c['C_matrix']), c['h'], tol=c['tol'])
        scale = max(np.abs(arr[f'{t}_{k}']).max() for k in STRAIN)
        err = max(np.abs(strain[k] - arr[f'{t}_{k}']).max() for k in STRAIN) / scale
        assert err < 1e-8, (t, err)
        assert info['converged'] and info['modes_dropped'] == c['modes_dropped']
        assert abs(info['iterations'] - c['iterations']) <= 1, (t, info, c['iterations'])


def test_oracle_fd_strain_matches_fig4_environment():
    meta, _ = _cases()
    f = meta['fig4']
    fx = np.load(os.path.join(GOLDEN, 'fig4_b6_fields.npz'))
    strain, info = ofd.solve_strain_fd(fx['mask'], f['eps_star'], tuple(f['C_dot']),
                                       tuple(f['C_matrix']), f['h'], tol=f['tol'])
    scale = max(np.abs(fx[k]).max() for k in STRAIN)
    err = max(np.abs(strain[k] - fx[k]).max() for k in STRAIN) / scale
    assert info['converged'] and err < 1e-8, err


def test_element_arrays_rigid_modes_and_symmetry():
    """K has the rigid translations in its null space (sum over b of K[a, b] = 0) and the
    symmetry K[a, b, j, l] = K[b, a, l, j] of a quadratic energy (elasticity_fd.py:156-176)."""
    K, W = ofd.element_arrays(83.29, 45.26, 39.59, 0.5)
    assert np.abs(K.sum(axis=1)).max() < 1e-12 * np.abs(K).max()
    assert np.abs(K - K.transpose(1, 0, 3, 2)).max() < 1e-12 * np.abs(K).max()
    assert np.abs(W.sum(axis=0)).max() < 1e-14
