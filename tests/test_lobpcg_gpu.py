"""GPU LOBPCG against the reference's scipy path: iterate by iterate, and solve by solve."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


@pytest.fixture(scope='module')
def small():
    z = np.load(os.path.join(GOLDEN, 'solve_cases.npz'))
    with open(os.path.join(GOLDEN, 'solve_cases.json')) as fh:
        meta = json.load(fh)
    shape = tuple(meta['shape'])
    f8 = {k[3:]: z[k] for k in z.files if k.startswith('f8_')}
    f4 = {k[3:]: z[k] for k in z.files if k.startswith('f4_')}
    return dict(z=z, meta=meta, shape=shape, h=float(z['h']), f8=f8, f4=f4, mask=z['mask'])


def _op(small, nb=8, hole=False):
    from qd3dsolver_b200 import kp_pryor as kpg
    f = small['f8'] if nb == 8 else small['f4']
    st = {k: f[k] for k in ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')}
    return kpg.confined_hamiltonian(kpg.GridOperators(small['shape'], small['h']), f, nb,
                                    hole_convention=hole, strain=st)


def _oracle_op(small, nb=8, hole=False):
    from oracle import kp_operator as ko
    f = small['f8'] if nb == 8 else small['f4']
    return ko.confined_hamiltonian(small['shape'], small['h'], f, nb, hole_convention=hole,
                                   strain=True)


def test_iterates_follow_scipy(small):
    """Same X0, same folded operator: residual histories agree over the first iterations."""
    import warnings
    import scipy.sparse.linalg as spla
    from qd3dsolver_b200 import eigensolvers as eg
    from oracle import eigensolvers as oe
    H = _op(small)
    Ho = _oracle_op(small)
    sigma = small['meta']['interior_cb']['sigma']
    X0 = oe.start_block(H.shape[0], 6, 0)
    lam, V, hist, info = eg.lobpcg_device(H, X0, folded=True, sigma=sigma, tol=1e-12,
                                          maxiter=12)
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        mu, Vo, ho = spla.lobpcg(oe.folded_operator(Ho, sigma), X0.copy(), largest=False,
                                 tol=1e-12, maxiter=12, retResidualNormsHistory=True)
    ho = np.array(ho)
    assert len(hist) == len(ho)
    rel = np.abs(hist[:8] - ho[:8]) / np.abs(ho[:8])
    assert rel.max() < 1e-6, rel.max()
    assert np.abs(lam - mu).max() < 1e-6 * np.abs(mu).max()


def test_solve_interior_matches_reference_cb_vb(small):
    from qd3dsolver_b200 import eigensolvers as eg
    H = _op(small)
    for band in ('cb', 'vb'):
        ref = small['meta']['interior_' + band]
        E, V, info = eg.solve_interior(H, k=ref['k'], sigma=ref['sigma'], tol=ref['tol'],
                                       maxiter=ref['maxiter'], verbose=False)
        assert np.abs(E - np.array(ref['E'])).max() < 1e-8, (band, E, ref['E'])
        assert info['residuals'].max() < 1e-8
        assert info['converged'] and info['status'] == 'converged'
        assert abs(info["iterations"] - ref["iterations"]) <= 0.25 * ref["iterations"]
        assert V.shape == (H.shape[0], ref['k']) and V.dtype == np.complex128
        G = V.conj().T @ V
        assert np.abs(G - np.eye(ref['k'])).max() < 1e-10
        from oracle import post
        lvl, _, worst = post.kramers_levels(E, post.localization(V, small['mask']))
        assert worst < 1e-7


def test_solve_lowest_four_band_hole(small):
    from qd3dsolver_b200 import eigensolvers as eg
    H = _op(small, nb=4, hole=True)
    ref = small['meta']['lowest_4band_hole']
    E, V, info = eg.solve_lowest(H, k=ref['k'], tol=ref['tol'], maxiter=ref['maxiter'],
                                 verbose=False)
    assert np.abs(E - np.array(ref['E'])).max() < 1e-8
    assert abs(info['gap_to_next'] - ref['gap_to_next']) < 1e-6
    assert info['residuals'].max() < 1e-8


def test_solve_lowest_hole_negates(small):
    """solve_lowest_hole(H) == reversed negation of solve_lowest(-H), checked with scipy."""
    import warnings
    import scipy.sparse.linalg as spla
    from qd3dsolver_b200 import eigensolvers as eg
    from oracle import eigensolvers as oe
    H = _op(small, nb=4, hole=False)
    Ho = _oracle_op(small, nb=4, hole=False)
    E, V, info = eg.solve_lowest_hole(H, k=4, tol=1e-9, maxiter=3000, verbose=False)
    Eo, Vo, io = oe.solve_lowest(-Ho, k=4, tol=1e-9, maxiter=3000)
    assert np.abs(E - (-Eo[::-1])).max() < 1e-8
    assert np.all(np.diff(E) >= 0)


def test_maxiter_status_and_best_iterate(small):
    from qd3dsolver_b200 import eigensolvers as eg
    H = _op(small)
    sigma = small['meta']['interior_cb']['sigma']
    E, V, info = eg.solve_interior(H, k=4, sigma=sigma, tol=1e-12, maxiter=5, verbose=False)
    assert info['status'] == 'maxiter'
    assert info['iterations'] <= 5 + 2
    assert not info['converged']


def test_residual_verification_layer(small):
    from qd3dsolver_b200 import eigensolvers as eg
    from oracle import eigensolvers as oe
    H = _op(small)
    Ho = _oracle_op(small)
    rng = np.random.default_rng(1)
    V = rng.standard_normal((H.shape[0], 3)) + 1j * rng.standard_normal((H.shape[0], 3))
    E = np.array([0.1, 0.5, 1.2])
    assert np.allclose(eg.residual_norms(H, E, V), oe.residual_norms(Ho, E, V), rtol=1e-12)
    assert np.allclose(eg.rayleigh_quotients(H, V), oe.rayleigh_quotients(Ho, V), rtol=1e-12)
    assert eg.hermiticity_error(H) < 1e-12


def test_small_problem_takes_the_dense_path(small):
    """Fewer than five block widths of rows: like scipy's lobpcg, the drop-ins warn and solve the
    dense eigenproblem (here on the device); energies equal the oracle operator's dense ones."""
    import warnings
    from qd3dsolver_b200 import eigensolvers as eg, kp_pryor as kpg
    from oracle import kp_operator as ko
    shape = (2, 2, 1)
    f = {k: np.ascontiguousarray(v[:2, :2, :1]) for k, v in small['f8'].items()}
    st = {k: f[k] for k in ('exx', 'eyy', 'ezz', 'exy', 'eyz', 'ezx')}
    H = kpg.confined_hamiltonian(kpg.GridOperators(shape, small['h']), f, 8, strain=st)
    Hd = ko.confined_hamiltonian(shape, small['h'], f, 8, strain=True).toarray()
    w = np.linalg.eigvalsh(0.5 * (Hd + Hd.conj().T))
    n = H.shape[0]
    assert n < 5 * 9
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter('always')
        E, V, info = eg.solve_lowest(H, k=6, verbose=False)
    assert any('dense eigensolver' in str(r.message) for r in rec)
    assert info['iterations'] == 0 and info['status'] == 'converged'
    assert np.abs(E - w[:6]).max() < 1e-10 * np.abs(w).max()
    assert info['residuals'].max() < 1e-9
    sigma = float(0.5 * (w[n // 2] + w[n // 2 + 1]) + 1e-3)
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        Ei, Vi, ii = eg.solve_interior(H, k=6, sigma=sigma, verbose=False)
    assert ii['iterations'] == 0
    near = np.sort(w[np.argsort(np.abs(w - sigma))[:6]])
    assert np.abs(Ei - near).max() < 1e-9 * np.abs(w).max()
    H.close()
